/*
 * isdf_c.h - C ABI of the B200 ISDF engine (libisdf_b200.so).
 *
 * Drop-in boundary for the GPU ISDF() entry point of LibISDF:
 *   void isdf::isdffunc::ISDF(double* d_psirow, Domain domain, int nocc,
 *        int nstate, int nv1, int nc1, int nv2, int nc2, int mu_points,
 *        double* d_thetaCol, int* piv, int KmeansMaxIter_ISDF, bool check)
 *   (reference include/isdf.hpp:37, src/common/isdf.cpp:132-209).
 * The C++ overloads with that exact signature live in include/isdf.hpp and
 * wrap isdf_solve() below.
 *
 * Conventions (same as the reference, README.md:246-260):
 *  - one rank, one GPU; the caller allocates and frees every buffer;
 *  - psi: device, Ng x nstate, column-major, ld = Ng, read only;
 *  - theta: device, Ng x mu, column-major, ld = Ng, fully written (columns
 *    past the effective mu are zero-filled);
 *  - piv: HOST int[Ng], fully written;
 *  - grid index g = ix + nx*(iy + ny*iz).
 * Every function returns ISDF_OK (0) or a negative ISDF_ERR_* code and never
 * throws or exits; isdf_last_error() gives a message for the calling thread.
 * All plain pointers; no CUDA or torch types appear in the signatures
 * (streams are passed as void*, a cudaStream_t, NULL = the library's own).
 */
#ifndef ISDF_C_H
#define ISDF_C_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ISDF_OK 0
#define ISDF_ERR_ARG (-1)         /* invalid argument */
#define ISDF_ERR_CUDA (-2)        /* CUDA runtime / launch failure */
#define ISDF_ERR_NOMEM (-3)       /* device allocation failed */
#define ISDF_ERR_NOT_SPD (-4)     /* C C^T + eps I not positive definite */
#define ISDF_ERR_TIMEOUT (-5)     /* a bounded device wait ran out */
#define ISDF_ERR_UNSUPPORTED (-6) /* shape or option outside what is built */
#define ISDF_ERR_CANCELLED (-7)   /* serving: request cancelled */
#define ISDF_ERR_BUSY (-8)        /* serving: queue full */
#define ISDF_ERR_COMM (-9)        /* sharded solve: a collective failed or a rank did not arrive */

#define ISDF_SELECT_KMEANS 0
#define ISDF_SELECT_QRCP 1

#define ISDF_PRECISION_FP64 0  /* the reference's FP64 method */
#define ISDF_PRECISION_MIXED 1 /* INT8-sliced tcgen05 GEMMs, FP64 Cholesky / inverse */

/* Layout-compatible with the numeric fields of the reference's Domain
 * (include/common/domain.hpp:8-36); the MPI communicators are not needed
 * at world size 1. */
typedef struct isdf_domain_t {
  double length[3];
  double pos_start[3];
  int num_grid[3];
  int num_grid_fine[3];
} isdf_domain_t;

typedef struct isdf_options_t {
  int precision;          /* ISDF_PRECISION_* (default FP64) */
  int refine_steps;       /* must be 0 (the default): FP64 iterative refinement of the
                             mixed form's theta solve is not built, because each step
                             would cost a full Ng x mu x mu product while the mixed
                             form's fitted densities are already within 1e-6 of FP64;
                             nonzero returns ISDF_ERR_UNSUPPORTED */
  double qrcp_oversample; /* QRCP sketch width = IRound(sqrt(f * mu)); reference 1.5 */
  long long qrcp_seed;    /* srand48 seed of the QRCP sketch; reference 41 */
  long long rand_seed;    /* >= 0: srand() before K-means (only its npt < mu branch
                             draws from rand()); < 0: keep the process state */
  void* stream;           /* cudaStream_t to run on; NULL = library stream */
  int mixed_slices;       /* mixed precision: base-254 INT8 digits per FP64 operand, 5..7 (default 6) */
  int kmeans_warm_start;  /* nonzero: K-means starts from the caller's previous pivots,
                             piv[0..mu), when piv[0] != piv[1] (an SCF loop passes the
                             piv of its last solve back in): those with a weight above
                             the filter threshold, topped up with the first kept grid
                             points not among them, as the reference's KMEAN does
                             (src/common/utility.cpp:725-749; its ISDF() zeroes piv
                             first, isdf.cpp:174-175, so there it never happens).
                             0 (default): piv is ignored on input, as in the reference */
  int reserved[6];
} isdf_options_t;

typedef struct isdf_report_t {
  int rk_requested;  /* mu used (mu_points or the default formula) */
  int rk_eff;        /* selected points after de-duplication */
  int kmeans_iters;  /* Lloyd iterations run (-1: early-return branch) */
  int npt;           /* grid points kept by the weight filter */
  double fit_err;    /* check: ||rho - theta C||_F / ||rho||_F */
  double coul_err;   /* check: relative truncated-Coulomb 4-index error */
  double t_select_ms;  /* wall time of weight + selection */
  double t_fit_ms;     /* wall time of the fit */
  double t_zct_ms;     /* device time of the Z C^T GEMM (CUDA events) */
  double t_chol_ms;    /* device time of C C^T + Cholesky */
  double t_solve_ms;   /* device time of the two triangular sweeps */
  double t_check_ms;
  double t_total_ms;
  int chol_info;       /* > 0: leading minor that failed */
  int kernel_launches; /* kernels this library launched for the solve */
  float t_gemm_ms;     /* GEMM launches of the triangular stage alone (FP64: the whole stage) */
  float kmeans_search_frac; /* share of K-means point assignments that ran the cell search */
  int qrcp_steps;           /* QRCP: pivots taken */
  int qrcp_norm_recomputes; /* QRCP: residual norms recomputed exactly because the
                               downdate lost accuracy (dgeqpf's cancellation test) */
  int kmeans_warm_pivots;   /* K-means warm start: previous pivots reused as initial
                               centroids (-1: cold start) */
  int reserved[1];
} isdf_report_t;

/* Fills *opt with the reference's defaults. */
void isdf_default_options(isdf_options_t* opt);

/* Full ISDF solve (reference src/common/isdf.cpp:132-209 ->
 * src/cuda/isdf-gpu.cpp:9-403, with the Kmeans/QRCP selector of the CPU entry
 * point src/common/isdf.cpp:60-74). mu_points = 0 selects
 * IRound(sqrt((nc1+nv1)(nc2+nv2)) * 8) (isdf.cpp:160-164). opt and rep may
 * be NULL. Synchronous: returns after theta and piv are written. */
int isdf_solve(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate, int nv1,
               int nc1, int nv2, int nc2, int mu_points, double* d_theta, int* piv,
               int kmeans_max_iter, int selector, int check, const isdf_options_t* opt,
               isdf_report_t* rep);

/* K-means weight w(r) = sum_{S2} psi^2 * sum_{S1} psi^2, bit-exact with the
 * reference CPU loop src/cpu/getpoints_Kmeans_MPI.cpp:33-45 (the GPU kernel
 * it replaces is calculateKmeansWeight, src/cuda/cuda_utils.cu:124-166,553-564).
 * d_w: device double[ng]. */
int isdf_kmeans_weight(const double* d_psi, long long ng, int nstate, int nocc, int nv1, int nc1,
                       int nv2, int nc2, double* d_w, void* stream);

/* K-means interpolation-point selection from a device weight vector
 * (reference KMEAN, src/common/utility.cpp:631-988). piv: host int[Ng]
 * (fully written); *rk_eff: distinct points selected; *iters: Lloyd
 * iterations run (-1 on the npt < mu early return). */
int isdf_kmeans_select(const isdf_domain_t* dom, const double* d_w, int mu, int max_iter,
                       long long rand_seed, int* piv, int* rk_eff, int* iters, int* npt,
                       void* stream);

/* No counterpart in the reference (one system per call): the K-means
 * selections of `count` small systems (Ng <= 2^20, mu <= 512, cold start) in
 * one cooperative launch, a group of CTAs per system; each result equals
 * isdf_kmeans_select()'s on the same input, bit for bit. Arrays of `count`:
 * doms, d_w (device weights), mu, max_iter, piv (host int[Ng] each, fully
 * written), rk_eff / iters / npt (outputs). rand_seed as in
 * isdf_kmeans_select (applied before each system). The serving loop batches
 * its small requests through this. */
int isdf_kmeans_select_batch(int count, const isdf_domain_t* doms, const double* const* d_w,
                             const int* mu, const int* max_iter, long long rand_seed,
                             int* const* piv, int* rk_eff, int* iters, int* npt, void* stream);

/* FP64 fit for given pivots (reference src/cuda/isdf-gpu.cpp:112-402 /
 * src/cpu/getbasis_MPI.cpp:9-250): theta = (Z C^T)(C C^T + eps I)^{-1} with
 * eps = 1e-10 tr(C C^T)/rk, Z C^T = (psi_S1 psi_S1(mu)^T) o (psi_S2 psi_S2(mu)^T).
 * piv: host int[>= rk], the first rk entries are the interpolation points.
 * d_theta: device Ng x rk, ld = Ng. *chol_info > 0 on a non-SPD matrix. */
int isdf_fit(const double* d_psi, long long ng, int nstate, int nocc, int nv1, int nc1, int nv2,
             int nc2, int rk, const int* piv, double* d_theta, int precision, int refine_steps,
             int* chol_info, void* stream);
/* (refine_steps must be 0; see isdf_options_t.refine_steps.) */

/* The check of the reference (src/common/checkcode.cpp:54-313, called by
 * src/common/isdf.cpp:193-206 when check = true): the pair-density fit error
 * ||rho - theta C||_F / ||rho||_F and the relative truncated-Coulomb (R = 5)
 * 4-index error of the ISDF form, here with cuFFT D2Z half spectra. The
 * reference prints both; here they are returned. Cost O(Ng * Npair^2), Npair =
 * (nv1+nc1)(nv2+nc2): sizes whose pair spectra exceed the device budget
 * return ISDF_ERR_UNSUPPORTED. piv: host, first rk entries used. */
int isdf_check(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate, int nv1,
               int nc1, int nv2, int nc2, int rk, const int* piv, const double* d_theta,
               double* fit_err, double* coul_err, void* stream);

/* No counterpart in the reference: its check (src/common/checkcode.cpp:54-313)
 * covers all Npair = (nv1+nc1)(nv2+nc2) pairs at O(Ng * Npair^2) and is out of
 * reach beyond the Si8-like size. This extension computes the same two errors
 * restricted to a caller-chosen list of state pairs (pair index
 * (k - (nocc-nv1)) * (nv2+nc2) + (j - (nocc-nv2)), the reference's numbering,
 * checkcode.cpp:62-73): the fit error ||rho - theta C||_F / ||rho||_F over all
 * grid points of those pairs, and the relative truncated-Coulomb error of the
 * pair block (ij|V|kl), ij, kl in the list, with the ISDF form evaluated from
 * the spectra of the fitted densities theta c_ij (by linearity of the FFT the
 * reference's c_ij^T Re(zeta^H V zeta) c_kl). With the list of all pairs it
 * gives isdf_check()'s numbers. pairs: host int[npair_sample], 1 <=
 * npair_sample <= 4096; piv: host, first rk entries used. */
int isdf_check_sampled(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate,
                       int nv1, int nc1, int nv2, int nc2, int rk, const int* piv,
                       const double* d_theta, int npair_sample, const int* pairs,
                       double* fit_err, double* coul_err, void* stream);

/* The ISDF Coulomb matrix A(mu, nu) = Re sum_G conj(zeta_mu(G)) V(G) zeta_nu(G),
 * zeta_mu the spectrum of theta column mu scaled by vol/Ng and V the
 * truncated Coulomb kernel of the check (R = 5): the matrix the reference's
 * check forms from theta (src/common/checkcode.cpp:249-288) and the operator a
 * GW / RPA / TDDFT code applies to interpolation-point quantities. d_theta:
 * device Ng x rk, ld = Ng (read only); d_A: device rk x rk, column-major.
 * Device memory: rk x 2 (nx/2+1) ny nz doubles of half spectra (Si216: 44 GB)
 * plus two 128-column transform buffers. */
int isdf_coulomb_matrix(const isdf_domain_t* dom, const double* d_theta, int rk, double* d_A,
                        void* stream);

/* Size of the fixed device scratch array behind isdf_fit_noalloc(). */
#define ISDF_NOALLOC_SCRATCH_BYTES (8u << 20)

/* No counterpart in the reference. isdf_fit() with every scratch array taken
 * from one fixed 8 MiB __device__ array inside the library instead of device
 * allocations: it calls no cudaMalloc / cudaFree and no allocating library
 * routine. For callers that cannot have the library allocate device memory
 * mid-run, e.g. a DFT host code that has reserved (nearly) all of HBM for its
 * own pool at start-up, or one that cannot afford the device-wide
 * synchronisation of cudaFree. The caller still passes psi, piv and theta.
 * Limit: the fit's scratch for (rk, nstate) must fit in 8 MiB (for example
 * rk <= 512 with nstate <= 512); larger sizes return ISDF_ERR_UNSUPPORTED
 * with a message naming the bytes needed. Every process that loads the
 * library holds the array on each GPU it uses until exit. All calls on a
 * device share the array, so calls that overlap on the GPU race; it keeps
 * the last call's contents (each call clears what must start at zero). Every
 * call looks up the array's device address on the current device (a cheap
 * runtime query, so the address stays right after cudaDeviceReset); the first
 * call on a device also loads the array's module, so make it before any
 * stream capture. stream NULL = the legacy default stream. Synchronous. */
int isdf_fit_noalloc(const double* d_psi, long long ng, int nstate, int nocc, int nv1, int nc1,
                     int nv2, int nc2, int rk, const int* piv, double* d_theta, int* chol_info,
                     void* stream);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference (one system per ISDF() call). A
 * continuous-batching server: requests for systems of any size arrive at any
 * time; `slots` solves run concurrently on their own streams (their kernels
 * overlap on the GPU); a request starts when its device workspace fits in
 * what the budget has left (small requests may pass a large head until it
 * has been passed `max_skips` times); the K-means selections of small
 * requests waiting together run in one launch (batch_small), their fits then
 * on the slots; psi / theta / piv stay the caller's buffers (device, device,
 * host) and must stay valid until the request is done. Results are the same
 * as isdf_solve() on the same request, bit for bit. */
typedef struct isdf_server_config_t {
  int device;              /* CUDA device of the server (default 0) */
  int slots;               /* concurrent solves (default 4) */
  size_t hbm_budget_bytes; /* workspace budget; 0 = half of the free memory at creation */
  int max_queue;           /* pending requests before submit returns ISDF_ERR_BUSY (4096) */
  int max_skips;           /* times a waiting head may be passed by smaller requests (64) */
  int batch_small;         /* small K-means requests (Ng <= 2^20, mu <= 512, cold start)
                              whose selections run together in one launch, at most this
                              many at a time (default 32; 0: each request on its own) */
  int reserved[3];
} isdf_server_config_t;

typedef struct isdf_request_t {
  isdf_domain_t dom;
  const double* d_psi;
  int nocc, nstate, nv1, nc1, nv2, nc2, mu_points;
  double* d_theta;
  int* piv;
  int kmeans_max_iter;
  int selector;
  int check;
  isdf_options_t opt; /* opt.stream is ignored: each slot has its own stream */
} isdf_request_t;

typedef struct isdf_server_stats_t {
  long long submitted, completed, failed, cancelled;
  double p50_ms, p99_ms, mean_ms; /* submit-to-completion latency of completed requests */
  double solves_per_s;            /* completed / (last completion - first submit) */
  int peak_concurrency, queued, running, reserved0;
  size_t peak_bytes; /* largest workspace total in use at once */
} isdf_server_stats_t;

void isdf_server_default_config(isdf_server_config_t* cfg);
int isdf_server_create(const isdf_server_config_t* cfg, void** server);
/* Queues a request; *ticket identifies it. ISDF_ERR_BUSY when the queue is full. */
int isdf_server_submit(void* server, const isdf_request_t* req, long long* ticket);
/* *state: 0 queued, 1 running, 2 done; *status: the solve's return code once done. */
int isdf_server_poll(void* server, long long ticket, int* state, int* status, isdf_report_t* rep);
/* Blocks until done (timeout_ms < 0: no limit; else ISDF_ERR_TIMEOUT when it runs out). */
int isdf_server_wait(void* server, long long ticket, double timeout_ms, int* status,
                     isdf_report_t* rep);
/* Removes a request that has not started (its status becomes ISDF_ERR_CANCELLED). */
int isdf_server_cancel(void* server, long long ticket);
int isdf_server_stats(void* server, isdf_server_stats_t* stats);
/* Cancels queued requests, waits for running ones, frees the server. */
int isdf_server_destroy(void* server);

/* ---------------------------------------------------------------- sharded
 * Grid-row sharding over several GPUs, one rank per GPU: the layout of the
 * reference's p-rank GPU ISDF() (src/common/isdf.cpp:132-188 ->
 * src/cuda/isdf-gpu.cpp:9-403). Rank r holds grid rows [start_r, start_r +
 * count_r) of psi, start_r = r (Ng / p) + min(r, Ng % p) and count_r = Ng / p +
 * (r < Ng % p) (isdf_row_block), as d_psirow (count_r x nstate, ld =
 * count_r). The ranks exchange the weights (an all-gather), run the
 * reference's p-rank KMEAN (each rank owns a block of the filtered point
 * list, folds its centroid sums in its point order; the partial sums are
 * combined in binomial-tree order, the order of MPICH's binomial reduce and
 * the only possible one at two ranks; the nearest point of each centroid is
 * the smallest distance over the ranks, ties to the smaller grid index, as
 * MPI_MINLOC), gather the psi rows at the pivots, and fit their own grid
 * rows (C C^T and its Cholesky factor are computed on every rank). piv (host
 * int[Ng]) is the same on every rank and equals the reference's p-rank piv bit
 * for bit (its one-rank piv in all but rare rounding and tie cases); theta's
 * rows are those of the one-rank solve with the same piv.
 *
 * theta layouts:
 *  ISDF_THETA_ROWS    d_theta = this rank's rows, count_r x mu, ld = count_r:
 *                     no exchange (the B200 form);
 *  ISDF_THETA_CYCLIC  the reference's d_thetaCol: Ng x w_r, ld = Ng, holding
 *                     theta's columns r, r + p, r + 2p, ... (w_r = mu / p +
 *                     (r < mu % p)), the layout GPU_AlltoallBackward produces
 *                     (src/common/utility.cpp:444-526); one all-to-all of theta.
 * Columns past the effective mu are zero in both. */
#define ISDF_THETA_ROWS 0
#define ISDF_THETA_CYCLIC 1

typedef struct isdf_comm isdf_comm_t;

/* Transport callbacks for callers with their own collectives (for instance a
 * CUDA-aware MPI: MPI_Allgatherv / MPI_Alltoallv on device buffers, after
 * synchronising `stream`). Sizes and displacements are in bytes, one entry per
 * rank. Return 0 on success. The operation must be complete, or ordered on
 * `stream`, when the callback returns. */
typedef struct isdf_comm_ops_t {
  int (*allgatherv)(void* ctx, const void* d_send, size_t send_bytes, void* d_recv,
                    const size_t* recv_bytes, const size_t* recv_displs, void* stream);
  int (*alltoallv)(void* ctx, const void* d_send, const size_t* send_bytes,
                   const size_t* send_displs, void* d_recv, const size_t* recv_bytes,
                   const size_t* recv_displs, void* stream);
} isdf_comm_ops_t;

/* NCCL transport (NCCL is opened at run time: libnccl.so.2). Rank 0 makes
 * the id, the caller hands it to every rank (any out-of-band channel), and
 * each rank, with its own GPU current, creates its communicator. */
int isdf_comm_nccl_unique_id(unsigned char id[128]);
int isdf_comm_create_nccl(const unsigned char id[128], int rank, int size, isdf_comm_t** comm);
/* `size` ranks inside this process (one host thread per rank calls the
 * sharded functions with its comms[r]); devices[r]: rank r's GPU (NULL: all on
 * the current device). A rank that does not reach a collective within
 * timeout_s seconds fails it with ISDF_ERR_COMM, and the group with it. */
int isdf_comm_create_local(int size, const int* devices, double timeout_s, isdf_comm_t** comms);
int isdf_comm_create_callbacks(const isdf_comm_ops_t* ops, void* ctx, int rank, int size,
                               isdf_comm_t** comm);
int isdf_comm_rank(const isdf_comm_t* comm, int* rank, int* size);
/* Fails this rank's outstanding and later collectives (NCCL: ncclCommAbort;
 * local group: the whole group). For failure handling. */
int isdf_comm_abort(isdf_comm_t* comm);
/* Frees the communicator and the rank's workspace. */
int isdf_comm_destroy(isdf_comm_t* comm);
/* The reference's row block of rank `rank`: start and count of n items. */
int isdf_row_block(long long n, int size, int rank, long long* start, long long* count);

/* The sharded ISDF solve (K-means selector, no check): every rank calls it
 * with the same arguments except d_psirow and d_theta. opt->stream: the
 * rank's stream (NULL: the communicator's own). opt->rand_seed (only the
 * npt < mu branch draws): each rank draws from its own copy of libc's rand()
 * sequence for that seed, a negative seed standing for 1, the state every
 * rank process of the reference starts from. Synchronous. */
int isdf_solve_sharded(isdf_comm_t* comm, const isdf_domain_t* dom, const double* d_psirow,
                       int nocc, int nstate, int nv1, int nc1, int nv2, int nc2, int mu_points,
                       double* d_theta, int theta_layout, int* piv, int kmeans_max_iter,
                       const isdf_options_t* opt, isdf_report_t* rep);

/* The p-rank K-means selection alone, from the full weight vector on every
 * rank (d_w: device double[Ng]); outputs as isdf_kmeans_select. */
int isdf_kmeans_select_sharded(isdf_comm_t* comm, const isdf_domain_t* dom, const double* d_w,
                               int mu, int max_iter, long long rand_seed, int* piv, int* rk_eff,
                               int* iters, int* npt);

/* Message for the last error on this thread ("" if none). */
const char* isdf_last_error(void);
const char* isdf_status_string(int code);

/* Device memory the solve needs beyond psi and theta, in bytes, for the
 * default QRCP oversampling (1.5) and WITHOUT the check's buffers (their size
 * depends on the grid's shape, which this signature does not carry): the
 * `check` argument is ignored. isdf_request_workspace_bytes() gives the full
 * footprint of one request. */
size_t isdf_workspace_bytes(long long ng, int nstate, int mu, int selector, int precision,
                            int check);

/* The full device footprint of one isdf_solve() call beyond psi and theta, in
 * bytes: the selector's, the fit's and (check != 0) the check's buffers for
 * this grid, state window, mu (0 = the default formula) and options (QRCP
 * oversampling, precision; opt may be NULL). The serving loop admits requests
 * by this figure. Returns 0 for invalid arguments. */
size_t isdf_request_workspace_bytes(const isdf_domain_t* dom, int nstate, int nv1, int nc1,
                                    int nv2, int nc2, int mu_points, int selector, int check,
                                    const isdf_options_t* opt);

/* Releases the per-device workspace cached by isdf_solve(). */
void isdf_release_workspace(void);

#ifdef __cplusplus
}
#endif

#endif /* ISDF_C_H */
