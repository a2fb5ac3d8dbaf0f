// Bump allocator over one device buffer: the solve carves every scratch array
// out of a single allocation so that no cudaMalloc happens between kernels.
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace isdf_b200 {

struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  size_t off = 0;
  bool counting = false;  // size pass: only advance the offset

  template <typename T>
  T* take(size_t n) {
    size_t bytes = (n * sizeof(T) + 255) & ~(size_t)255;
    T* p = counting ? nullptr : reinterpret_cast<T*>(base + off);
    off += bytes;
    return p;
  }
  bool overflowed() const { return !counting && off > cap; }
};

}  // namespace isdf_b200
