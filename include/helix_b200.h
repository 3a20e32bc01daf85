/* helix_b200 — C ABI of the B200 HEOM propagator.
 *
 * This is the drop-in boundary for the reference's propagation path
 * (HELIX: helix::HEOMSolver().run(system, hierarchy, options) -> RunResult).
 * Plain C types only: pointers, sizes and status codes.  The C++ helix:: API
 * in include/helix/ is a thin layer over these entry points, and Python binds
 * them with ctypes (helix_b200/capi.py).
 *
 * Conventions
 *  - Every function returns HX_OK (0) or 1 + the helix::StatusCode value of
 *    the failure (include/helix/types.h; codes are append-only).  The text of
 *    the last failure on the calling thread is hx_last_error().
 *  - Complex buffers are interleaved (re, im) doubles, matrices row-major.
 *  - A context owns all device memory it uses and runs its work on one CUDA
 *    stream (hx_ctx_set_stream can substitute the caller's stream).  A
 *    context may be driven by one host thread at a time; several contexts
 *    may live on one device.
 *  - Hierarchy truncation uses the reference semantics: index vectors n with
 *    sum(n) < max_depth (exclusive bound; depth L <=> max_depth = L + 1).
 *  - Mode order is bath-major: mode = sum_{i<j}(K_i + 1) + k, k = 0 the Drude
 *    mode of bath j, k >= 1 its Pade modes.
 */
#ifndef HELIX_B200_H
#define HELIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HX_OK 0
/* 1 + helix::StatusCode (include/helix/types.h) */
#define HX_ERR_INVALID_DIMENSION 1
#define HX_ERR_INVALID_RUNTIME_OPTION 6
#define HX_ERR_UNSUPPORTED_PRECISION 7
#define HX_ERR_UNSUPPORTED_EXECUTION 10
#define HX_ERR_UNSUPPORTED_BATH 11
#define HX_ERR_UNSUPPORTED_HIERARCHY 12
#define HX_ERR_BATH_EXPONENTS_INVALID 14
#define HX_ERR_CUDA 15          /* StatusCode::CudaFailure (appended) */
#define HX_ERR_OUT_OF_MEMORY 16 /* StatusCode::OutOfMemory (appended) */
#define HX_ERR_NON_FINITE 17    /* StatusCode::NonFiniteState (appended) */
#define HX_ERR_DEVICE_TIMEOUT 18 /* StatusCode::DeviceWaitTimeout (appended) */

#define HX_PRECISION_SINGLE 0
#define HX_PRECISION_DOUBLE 1
/* Mixed precision: complex64 hierarchy state and single-precision
 * right-hand side, the tier-0 ADO (the reduced density matrix), its energy and
 * trace in double precision.  Needs 128 <= dim <= 1024, diagonal coupling
 * operators and max_depth >= 3.  No counterpart in the reference, whose
 * precision is fixed at compile time (src/legacy_compile_options.h:6). */
#define HX_PRECISION_MIXED 2

/* A sparse d x d complex operator in compressed rows: row r holds the entries
 * row_ptr[r] .. row_ptr[r+1]-1, entry p in column col[p] with value
 * val[2p] + i val[2p+1].  (The reference's SparseOperator,
 * include/helix/types.h:122-128, with 32-bit indices.) */
typedef struct hx_csr {
    const int32_t* row_ptr;     /* d + 1 */
    const int32_t* col;         /* nnz */
    const double* val;          /* 2 nnz */
    uint32_t nnz;
} hx_csr;

/* One Drude-Lorentz bath with Pade terms, coupled through the system operator
 * V_j = diag(coupling_diag) + sum_i coupling_flip[i] * sigma_x(spin i).
 * Replaces the compiled bath and coupling operator of the reference
 * (src/parameters.cu:25-31; buildSparseOperators, src/initialize.cu:95-147;
 * Bath, include/helix/types.h:108-128). */
typedef struct hx_bath {
    double inverse_temperature; /* beta (Param::Betah) */
    double damping;             /* gamma (Param::Gamma) */
    double coupling_strength;   /* zeta (Param::Zeta); lambda = zeta*gamma/2 */
    uint32_t pade_terms;        /* K (Param::KMax) */
    const double* coupling_diag; /* dim real values: diagonal of V_j */
    const double* coupling_flip; /* log2(dim) real values (sigma_x weights of V_j), or NULL */
    const hx_csr* coupling_csr;  /* or NULL; a general Hermitian V_j, in place of coupling_diag / _flip */
} hx_bath;

/* One HEOM problem.  H = diag(h_diag) + sum_i h_flip[i] * sigma_x(spin i),
 * spin i <-> bit i of the basis index.  Replaces initialize()
 * (src/initialize.cu:342-353) and the compiled parameters it reads. */
typedef struct hx_problem {
    uint32_t dim;               /* Hilbert dimension d = 2^spins, 2 <= d <= 4096 */
    const double* h_diag;       /* d diagonal entries of H */
    const double* h_flip;       /* log2(d) transverse-field coefficients, or NULL */
    uint32_t n_baths;
    const hx_bath* baths;
    uint32_t max_depth;         /* exclusive bound on sum(n) */
    double time_step;           /* dt (Param::Step) */
    uint32_t integration_order; /* Taylor order (Param::IntegrationNum), 1..8 */
    uint32_t precision;         /* HX_PRECISION_DOUBLE or HX_PRECISION_MIXED */
    uint32_t flags;             /* 0, HX_FLAG_FULL_STATE, HX_FLAG_DENSE_H */
    const hx_csr* h_csr;        /* or NULL; a general Hermitian H, in place of h_diag / h_flip */
} hx_problem;

/* General sparse operators (h_csr, coupling_csr; the reference validates
 * System::from_sparse but does not execute it, src/helix.cpp:166-258,335-347)
 * run on a two-pass stage that gathers along the CSR rows of H and V_j
 * (d <= 4096, double precision, full slabs).  Both must be Hermitian to 1e-12
 * of their largest entry; batches, closures, mixed precision and
 * hx_rhs_noalloc take diagonal / flip operators only. */

/* Every ADO of this hierarchy stays Hermitian (H and the V_j are Hermitian
 * and every term of the right-hand side maps Hermitian matrices to Hermitian
 * matrices), so for d = 32 ... 1024 with diagonal coupling operators (the
 * fused and band paths) the device state (complex64 in mixed precision) keeps
 * the upper triangle of each slab only (d(d+1)/2 elements instead of d^2),
 * which halves the memory traffic of a step; the flip and CSR paths keep
 * full slabs.  The C ABI still reads and writes full d x d
 * slabs; hx_ctx_write_state then rejects non-Hermitian ADOs.  This flag keeps
 * full slabs on the device, for general (non-Hermitian) states. */
#define HX_FLAG_FULL_STATE 1u
/* hx_problem.flags: evaluate the Hamiltonian commutator -i[H, u_n] of every
 * ADO as matrix products on the tensor cores (tcgen05, TF32 operands in a
 * 3-term split product, FP32 accumulation), for a general dense Hermitian H
 * (h_csr with any number of entries per row, or h_diag / h_flip).  The real
 * diagonal of H stays in the exact elementwise term, and ADO 0 (rho_0) takes
 * its product in FP64.  Needs
 * HX_PRECISION_MIXED, HX_FLAG_FULL_STATE, diagonal coupling operators and
 * 128 <= dim <= 1024; the states must be Hermitian (hx_ctx_write_state
 * checks).  No counterpart in the reference, whose H is diagonal
 * (src/legacy_compile_options.h:3) or applied as a sparse product. */
#define HX_FLAG_DENSE_H 2u

typedef struct hx_info {
    uint32_t dim;
    uint32_t modes;
    uint64_t hierarchy_size;    /* number of ADOs */
    uint64_t state_bytes;       /* device bytes of one hierarchy state (packed slabs count d(d+1)/2) */
    uint64_t device_bytes;      /* device memory the context holds */
    uint64_t steps_done;
    double time;                /* steps_done * dt */
    uint32_t kernels_per_step;  /* kernel launches one step enqueues */
    uint32_t stage_path;        /* HX_PATH_*: the stage kernels this context runs */
} hx_info;

/* hx_info.stage_path.  Sparse operators (hx_csr) that are a real diagonal
 * plus single-spin flips of one weight per spin are rewritten in that form
 * at creation and take the flip, fused or band path. */
#define HX_PATH_GENERIC 0u  /* stage_kernel: d <= 64 outside the fused shapes */
#define HX_PATH_FUSED 1u    /* herm_kernel / fused_kernel (+ upterm_kernel): d = 32, 64 */
#define HX_PATH_BAND 2u     /* band kernels: 128 <= d <= 1024, diagonal couplings */
#define HX_PATH_FLIP 3u     /* comm_kernel + combine_kernel: couplings with spin flips */
#define HX_PATH_CSR 4u      /* csr_comm_kernel + csr_combine_kernel: general sparse operators */
#define HX_PATH_SMALL 5u    /* small_kernel: d <= 16 with sigma_z couplings (batched neighbour gathers) */
#define HX_PATH_DENSE 6u    /* HX_FLAG_DENSE_H: tc_split_gemm_kernel + zgemm_kernel + band kernels */

/* Profiling counters (replaces src/library/backend_profiling.cpp:9-137). */
typedef struct hx_counters {
    uint64_t kernel_launches;
    uint64_t stage_launches;
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
} hx_counters;

typedef struct hx_ctx hx_ctx;

/* Text of the last failure on this thread ("" if none). */
const char* hx_last_error(void);

/* Library version string. (helix::runtimeVersion, src/helix.cpp:18-21) */
const char* hx_version(void);

/* Make `device` the calling thread's current CUDA device (contexts are
 * created on the current device).  (cudaSetDevice in Context::Impl,
 * src/helix.cpp:568-573) */
int hx_select_device(int device);

/* Number of ADOs for `modes` modes and exclusive depth bound `max_depth`.
 * (hierarchySizeFor, src/initialize_detail.h:159-172) */
int hx_hierarchy_size(uint32_t modes, uint32_t max_depth, uint64_t* count);

/* Hierarchy index rows (count x modes) and neighbour edges (count x 2*modes)
 * in the reference order and sentinel convention, built on the device and
 * copied to the caller's host buffers: rows in lexicographic order with mode
 * 0 most significant, edges[i][k] = index of n_i + e_k, edges[i][modes + k] =
 * index of n_i - e_k, sentinel = count.  `count` must equal
 * hx_hierarchy_size().  (buildHierarchyRows / buildHierarchyEdges,
 * src/initialize_detail.h:174-269; initializeHierarchyStorage,
 * src/initialize.cu:237-250) */
int hx_hierarchy_tables(uint32_t modes, uint32_t max_depth, int32_t* rows, int32_t* edges,
                        uint64_t count);

/* Pade poles xi_k and residues eta_k (k < K) of the Bose function, [K-1/K].
 * (getPsdPoleResidue, src/psd/psd.cu:12-113) */
int hx_psd(uint32_t K, double* poles, double* residues);

/* Seeded J_ij ~ N(0,1) for i<j in row-major pair order (splitmix64 +
 * Box-Muller), written symmetric into J (n x n, zero diagonal).  Synthetic
 * instance generator; no counterpart in the reference. */
int hx_seeded_couplings(uint32_t n_spins, uint64_t seed, double* J);

/* Create a context on the current CUDA device: builds tables and
 * coefficients on the device, allocates the state and sets rho to the
 * reference initial state |d-1><d-1| with all other ADOs zero.
 * (initialize(), src/initialize.cu:342-353; LegacyRuntimeSession::create,
 * src/library/legacy_runtime_session.cu:53-77) */
int hx_ctx_create(const hx_problem* problem, hx_ctx** out);

/* Release every device resource of the context.
 * (LegacyRuntimeSession::destroy, src/library/legacy_runtime_session.cu:108-118;
 * clearLiouvilleStorage, src/liouville.cu:871-920) */
void hx_ctx_destroy(hx_ctx* ctx);

/* Use `stream` (a cudaStream_t; NULL = the context's own stream) for all
 * further work of the context. */
int hx_ctx_set_stream(hx_ctx* ctx, void* stream);
int hx_ctx_get_stream(hx_ctx* ctx, void** stream);

int hx_ctx_info(const hx_ctx* ctx, hx_info* info);
int hx_ctx_counters(const hx_ctx* ctx, hx_counters* counters);

/* Enqueue `nsteps` integrator steps on the context stream (asynchronous).
 * (develop() loop, src/liouville.cu:502-590;
 * LegacyRuntimeSession::run_steps, src/library/legacy_runtime_session.cu:79-100) */
int hx_ctx_step(hx_ctx* ctx, uint64_t nsteps);

/* As hx_ctx_step, and after every step write rho_0 (d*d complex) to
 * rho0_trace[step] and Tr(H rho_0) to energy_trace[step] (either may be NULL).
 * Host buffers; the call returns when the last values have landed.
 * (ResultMode::ObservableTrace, validation-only in the reference,
 * src/helix.cpp:315-319; energy as in src/cli_compatibility.cu:80-98) */
int hx_ctx_step_trace(hx_ctx* ctx, uint64_t nsteps, double* rho0_trace, double* energy_trace);

/* Wait for all work of the context. */
int hx_ctx_sync(hx_ctx* ctx);

/* Copy rho_0 (d*d complex, row-major) into a host buffer of n doubles
 * (n >= 2*d*d).  (ResultExtractor::final_reduced_density,
 * src/library/result_extractor.cu:35-90) */
int hx_ctx_read_rho0(hx_ctx* ctx, double* out, uint64_t n);

/* Tr(H rho_0) and Tr(rho_0) computed on the device.
 * (energyFromDensityDiagonal, src/library/energy_observable.cpp:8-39,
 * generalised to the off-diagonal H) */
int hx_ctx_observables(hx_ctx* ctx, double* energy, double* trace_re, double* trace_im);

/* Full hierarchy state (hierarchy_size * d * d complex) to / from host
 * memory, reference ADO order.  (snapshot writer / loader,
 * src/cli_compatibility.cu:130-145, src/initialize.cu:266-285) */
int hx_ctx_read_state(hx_ctx* ctx, double* out, uint64_t n);
int hx_ctx_write_state(hx_ctx* ctx, const double* in, uint64_t n);

/* Whole state to / from a file in the reference's snapshot format
 * (snapshot_rho<N>.dat, src/cli_compatibility.cu:130-145, loader
 * src/initialize.cu:266-285): hierarchy_size * d * d complex values in ADO
 * order, row-major slabs, each value as its real then its imaginary part, in
 * float (real_bytes = 4, the reference's default compiled precision) or
 * double (8), native byte order, no header.  Loading checks the file size.
 * On a context with Hermitian-packed slabs loading keeps the Hermitian part of
 * each ADO and rejects an ADO whose anti-Hermitian part exceeds 1e-5 of its
 * largest element (single-precision snapshots of another program are
 * Hermitian to their rounding only). */
int hx_ctx_save_snapshot(hx_ctx* ctx, const char* path, uint32_t real_bytes);
int hx_ctx_load_snapshot(hx_ctx* ctx, const char* path, uint32_t real_bytes);

/* Energy trace in the reference CLI's outputEnergy.txt format
 * (src/cli_compatibility.cu:80-98): one line "time energy" per entry, both
 * with 8 significant digits.  Host only. */
int hx_write_energy_trace(const char* path, const double* times, const double* energies, uint64_t n);

/* Device pointer of the state (hierarchy_size * d * d double2), for callers
 * that fill or read it on the device.  In mixed precision this is the
 * double-precision slab of ADO 0 only (d * d double2).  With Hermitian-packed
 * slabs (32 <= d <= 1024, without HX_FLAG_FULL_STATE) each slab holds d(d+1)/2
 * double2: element (r, c), r <= c, at r*(d+1) + c - r when r < d/2, else at
 * (d-1-r)*(d+1) + c + 1. */
int hx_ctx_state_device_ptr(hx_ctx* ctx, void** ptr);

/* One evaluation of the right-hand side L(rho) of the current state into a
 * host buffer (hierarchy_size * d * d complex).  Test hook for parity of the
 * fused kernel against the reference RHS (getdRhoSparse, src/liouville.cu:749-869). */
int hx_ctx_rhs(hx_ctx* ctx, double* out, uint64_t n);

/* Enqueue `count` evaluations of the tensor-core product Y = X H_off of an
 * HX_FLAG_DENSE_H context (tc_split_gemm_kernel, the first kernel of every
 * stage) on its stream, on the current state and without changing it: the
 * entry exists to time and profile the product alone.
 * HX_ERR_UNSUPPORTED_EXECUTION for other contexts.  No counterpart in the
 * reference. */
int hx_ctx_dense_product(hx_ctx* ctx, uint32_t count);

/* Failure-detection test hook: the next step of a context whose steps run as
 * one cooperative launch (small slabs) waits at its first grid barrier for an
 * arrival that never comes, with a short poll limit.  The kernel gives up,
 * sets the device error word and returns before writing rho; the next
 * hx_ctx_sync reports HX_ERR_DEVICE_TIMEOUT, clears the error and the barrier
 * counter, and the context steps on from the state before the failed step.
 * HX_ERR_UNSUPPORTED_EXECUTION for other contexts.  No counterpart in the
 * reference. */
int hx_ctx_inject_wait_timeout(hx_ctx* ctx);

/* Device check that the state holds only finite values; returns
 * HX_ERR_NON_FINITE otherwise. */
int hx_ctx_check_finite(hx_ctx* ctx);

/* ------------------------------------------------------------------------
 * Batches: many independent instances in one persistent launch per stage.
 * The reference runs one instance per HEOMSolver::run (src/helix.cpp:723-772)
 * and has no batched mode; a batch is that call for hundreds of disorder
 * realisations of uneven size at once, with the disorder average of
 * <sigma_z(spin)> reduced on the device every step.
 * ------------------------------------------------------------------------ */
typedef struct hx_batch hx_batch;

typedef struct hx_batch_options {
    uint32_t observable_spin; /* spin whose <sigma_z> is averaged (bit index), default 0 */
    uint32_t tune;            /* 1 = run the tile-shape autotuner at creation */
    uint32_t tile_elems;      /* elements per tile (power of two, 64..8192); 0 = 2048 */
    uint32_t threads;         /* threads per CTA (multiple of 32, 64..1024); 0 = 256 */
} hx_batch_options;

typedef struct hx_batch_stats {
    uint32_t count;           /* instances */
    uint32_t tile_elems;
    uint64_t total_ados;
    uint64_t state_bytes;     /* bytes of one state of all instances */
    uint64_t device_bytes;
    uint64_t steps_done;
    uint64_t kernel_launches; /* kernels launched by stepping and tuning so far */
    uint32_t threads;
    uint32_t tiles;
    uint32_t grid;            /* persistent CTAs per stage launch */
    uint32_t kernels_per_step;
} hx_batch_stats;

/* Create a batch from `count` problems on the current device.  Every problem
 * has 2 <= dim <= 64, diagonal coupling operators, at most 64 modes, and all
 * share time_step and integration_order; each starts in |d-1><d-1|. */
int hx_batch_create(const hx_problem* problems, uint32_t count, const hx_batch_options* options,
                    hx_batch** out);
void hx_batch_destroy(hx_batch* batch);
int hx_batch_set_stream(hx_batch* batch, void* stream);
int hx_batch_info(const hx_batch* batch, hx_batch_stats* info);

/* Time every candidate tile shape on this batch (three stage launches each,
 * the state untouched) and keep the fastest; reports the choice. */
int hx_batch_tune(hx_batch* batch, uint32_t* tile_elems, uint32_t* threads);

/* Advance every instance `nsteps` steps (a captured CUDA graph per step).
 * If sz_sum_trace is not NULL, sz_sum_trace[t] receives, after step t, the
 * sum over instances of Tr(sigma_z(spin) rho_0) (divide by the instance count
 * for the disorder average; sums add across batches on several GPUs) and the
 * call returns when they have landed; otherwise it returns at once. */
int hx_batch_step(hx_batch* batch, uint64_t nsteps, double* sz_sum_trace);
int hx_batch_sync(hx_batch* batch);

/* rho_0 of one instance (d*d complex, row-major) into a host buffer of n doubles. */
int hx_batch_read_rho0(hx_batch* batch, uint32_t instance, double* out, uint64_t n);

/* ------------------------------------------------------------------------
 * Learned closure of a truncated hierarchy.  The reference truncates at
 * Param::JMax and drops the next tier (src/parameters.cu:31,
 * src/initialize_detail.h:196-213); a closure supplies, for every ADO n of the
 * top tier and every mode k, a prediction of the dropped up neighbour
 * rho_{n+e_k}, elementwise and linear in rho_n:
 *   rho_{n+e_k}(r, c) ~ A(k, n_k, r, c) rho_n(r, c),
 * the complex coefficient A given by a small MLP (BF16 weights, FP32
 * accumulation) from the features of (k, n_k, r, c): one-hot k, the coupling
 * diagonal of k's bath at r and at c, (E_r - E_c) scaled by the spread of the
 * diagonal of H, one-hot n_k.  The network is trained on the device from
 * deeper (fine) hierarchies; its Hermitian part, evaluated once into a table,
 * is what the stages apply.  No counterpart in the reference.
 * ------------------------------------------------------------------------ */
typedef struct hx_mlp hx_mlp;

/* in -> hidden -> GELU -> hidden -> GELU -> out; weights uniform(+-sqrt(6/fan_in))
 * from splitmix64(seed), biases zero. */
int hx_mlp_create(uint32_t in_dim, uint32_t hidden, uint32_t out_dim, uint64_t seed, hx_mlp** out);
void hx_mlp_destroy(hx_mlp* mlp);
/* Parameters as one FP32 array: W1 [hidden][in], b1, W2 [hidden][hidden], b2,
 * W3 [out][hidden], b3.  Setting them resets the optimiser. */
int hx_mlp_num_params(const hx_mlp* mlp, uint64_t* count);
int hx_mlp_get_params(hx_mlp* mlp, float* params, uint64_t count);
int hx_mlp_set_params(hx_mlp* mlp, const float* params, uint64_t count);
/* y[rows][out] = MLP(x[rows][in]) (host buffers; x is rounded to BF16). */
int hx_mlp_forward(hx_mlp* mlp, const float* x, uint32_t rows, float* y);
/* Mean-squared-error loss of MLP(x) against t and its gradient with respect
 * to every parameter (host buffers; layout as the parameters). */
int hx_mlp_gradients(hx_mlp* mlp, const float* x, const float* t, uint32_t rows, float* loss, float* grads,
                     uint64_t count);
/* Adam (lr, 0.9, 0.999, 1e-8) on minibatches of `batch` rows drawn from
 * (x, t) by splitmix64(seed + iteration); loss_trace[iters] may be NULL. */
int hx_mlp_train(hx_mlp* mlp, const float* x, const float* t, uint32_t rows, uint32_t batch, uint32_t iters,
                 float lr, uint64_t seed, float* loss_trace);

typedef struct hx_closure hx_closure;

/* Closure for the truncated (coarse) problem `coarse` (2 <= dim <= 64,
 * max_depth >= 2, diagonal coupling operators), trained from fine hierarchies
 * of the same system with max_depth = fine_max_depth; the training set holds
 * up to `capacity` snapshots on the device.  The MLP maps modes + 3 +
 * max_depth features through two GELU layers of width `hidden` to the two
 * reals of A. */
int hx_closure_create(const hx_problem* coarse, uint32_t fine_max_depth, uint32_t hidden, uint32_t capacity,
                      uint64_t seed, hx_closure** out);
void hx_closure_destroy(hx_closure* closure);
int hx_closure_mlp(hx_closure* closure, hx_mlp** mlp);
int hx_closure_info(const hx_closure* closure, uint32_t* top_ados, uint32_t* up_ados, uint32_t* snapshots,
                    double* s_in, double* s_out);
/* Add one snapshot from the current state of a fine-hierarchy context: the
 * coarse top-tier ADOs and their up neighbours. */
int hx_closure_harvest(hx_closure* closure, hx_ctx* fine);
/* Train on the snapshots: minibatches of `batch` elements (snapshot, top-tier
 * ADO, mode, element with a nonzero commutator weight), loss mean |A x - t|^2
 * with x, t scaled by their RMS over the set (fixed at the first call),
 * cosine-decayed Adam; then rebuild the coefficient table. */
int hx_closure_train(hx_closure* closure, uint32_t iters, uint32_t batch, float lr, uint64_t seed,
                     float* loss_trace);
/* Scales of a closure whose parameters were set from elsewhere. */
int hx_closure_set_scales(hx_closure* closure, double s_in, double s_out);
/* Every stage of `ctx` (the coarse problem) adds the closure term; NULL
 * detaches.  The closure must outlive its use. */
int hx_ctx_set_closure(hx_ctx* ctx, hx_closure* closure);

/* One evaluation of the right-hand side, drho = L(rho) for every ADO, that
 * allocates no memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc while they run this library (a host
 * framework that owns every byte of device memory through its own pool, or a
 * process at its device-memory budget): they pass the state `rho_device` and
 * the result `drho_device` (each hierarchy_size * dim * dim complex doubles,
 * full row-major slabs, device memory they already own, 16-byte aligned, not
 * overlapping) and the stream to run on (NULL = the legacy default stream;
 * it must belong to the current device).  The working tables live in one
 * fixed 8 MiB device array compiled into the library, reserved on every GPU
 * that loads it until the process exits; a problem whose tables need more is
 * rejected with HX_ERR_UNSUPPORTED_HIERARCHY and a message giving the size
 * needed.  The first call on a device looks up that array's device address
 * and caches it: make that first call before any stream capture, and make no
 * call on a device after cudaDeviceReset of it.  All calls share the array
 * (each call rewrites the tables and clears the error word), so calls that
 * overlap on the GPU race.  The call synchronizes `stream` and returns when
 * the result is complete. */
int hx_rhs_noalloc(const hx_problem* problem, const double* rho_device, double* drho_device, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HELIX_B200_H */
