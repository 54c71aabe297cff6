/*
 * qumasun_b200.h -- C ABI of the B200 Kohn-Sham H|psi> + LOBPCG engine.
 *
 * Plain C: opaque handles, integer status returns, plain pointers and sizes.
 * Every entry point returns QG_OK (0) or a negative qg_status. Nothing here
 * falls back to the CPU: without a usable CUDA device every call that needs
 * one returns QG_ERR_CUDA.
 *
 * Layout contract (same as the reference, so its buffers copy in without a
 * transpose): one state is an x-fastest grid array, index ix + nx*(iy + ny*iz);
 * a block of states is state-major, state s at X + s*ldx (ldx >= nx*ny*nz).
 * Complex (k-point) states follow the reference's per-state split layout
 * {re[N], im[N]} (lobpcg_z_multi_mpi.h:1005-1012): state s holds its real part
 * at X + s*ldx and its imaginary part at X + s*ldx + N, with ldx >= 2N.
 */
#ifndef QUMASUN_B200_H
#define QUMASUN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QG_API_VERSION 1

typedef enum qg_status {
    QG_OK = 0,
    QG_ERR_INVALID = -1,       /* bad argument */
    QG_ERR_CUDA = -2,          /* CUDA runtime error or no device */
    QG_ERR_NOMEM = -3,         /* device allocation failed */
    QG_ERR_CHOLESKY = -4,      /* Gram matrix B not positive definite */
    QG_ERR_TIMEOUT = -5,       /* a bounded device wait gave up */
    QG_ERR_NONFINITE = -6,     /* NaN/Inf met in inputs or iterates */
    QG_ERR_UNSUPPORTED = -7,   /* shape or option this build does not handle */
    QG_ERR_LIBRARY = -8,       /* cuBLAS / cuSOLVER / cuFFT error */
    QG_ERR_NOT_CONVERGED = -9  /* solver hit its iteration limit (results still written) */
} qg_status;

/* QG_MIXED_BF16X3 (LOBPCG only): the Gram products run on the library's tcgen05
 * kernel with every FP64 value split into 3 bfloat16 pieces (6 products, FP32
 * accumulation over one 64-row K block, FP64 across blocks; rows not a multiple of
 * 8 use cuBLAS BF16 GEMMs on 2 pieces) until the residual falls below 1e-6 or stops
 * halving, then as FP64; H, residuals, rotations, norms and the small eigensolves
 * stay FP64 throughout (a solve that reaches the tolerance or max_iter while still
 * mixed takes an FP64 Rayleigh-Ritz on X before its residuals are judged).
 * QG_FP64_INT8 (LOBPCG, real states): an FP64 iteration whose Gram products (pencils of
 * more than 128 columns) run on the tensor cores' int8 path: each column scaled by a
 * power of two and cut into 7 exact 7-bit slices, the 28 slice products with exact int32
 * accumulation, the scale groups added in FP64 -- as accurate as DGEMM (no counterpart in
 * the reference, whose Gram products are BLAS DGEMMs). */
typedef enum qg_precision { QG_FP64 = 0, QG_FP32 = 1, QG_MIXED_BF16X3 = 2, QG_FP64_INT8 = 3 } qg_precision;

typedef struct qg_context_s* qg_context;
typedef struct qg_hamiltonian_s* qg_hamiltonian;
typedef struct qg_learned_s* qg_learned;

/*
 * Hamiltonian description. The projector tables are the reference's own
 * per-atom cube form (PP_nonlocal_each_atom, PseudoPotOperator.h:21-24), as
 * tabulated by UpdatePosition (PseudoPotOperator.h:453-466):
 *  - projector k of atom a lives on the cube cube[6*(a*n_proj+k) + 0..5] =
 *    {begin_x, begin_y, begin_z, size_x, size_y, size_z} (GridForSphere,
 *    GridSubgrid.h:482-492; begins may be negative, the grid is periodic),
 *    values w_data[w_off[a*n_proj+k] + ...] x-fastest;
 *  - Y_lm of atom a, lm = l*l + (m + l), lives on the cube of the first
 *    projector with that l, values ylm_data[ylm_off[a*n_lm+lm] + ...].
 * The operator applied is the reference's mHamiltonianMatrix_ddm
 * (qumasun_mpi.matrix.h:20-43, kpoint: qumasun_kpoint.matrix.h:25-50):
 *   H psi = V psi + sum_atoms sum_k E_k sum_m |p_km> dV <p_km|psi> - 1/2 Lap psi
 * with p_k0 = w_k * Y00 for l = 0 and p_km = w_k * Y_lm for l >= 1
 * (ProjectionPP, PseudoPotOperator.h:740-772).
 * g = (gx, gy, gz) is the Bloch vector in bohr^-1 for the k-point operator
 * -(1/2)(Lap + 2i g.grad - g^2) (GridDifferenceKpoint8th.h:18-122); it is only
 * used by the complex entry points and must be zero for the real ones.
 * All pointers are HOST pointers; the library copies what it needs.
 */
typedef struct qg_hamiltonian_desc {
    int nx, ny, nz;
    double hx, hy, hz;
    int fd_order;              /* 2, 4 (the reference's composed 7-point stencil), 6, 8 */
    const double* V;           /* nx*ny*nz local potential (Ha) */
    int n_atoms;
    const double* atom_pos;    /* 3*n_atoms (bohr), informational */
    int n_proj;                /* projectors per atom (0 = no nonlocal term) */
    const int* proj_l;         /* n_proj angular momenta, 0..3 */
    const double* proj_E;      /* n_proj energies E_k (Ha) */
    const int* cube;           /* 6*n_atoms*n_proj */
    const double* w_data;
    const long long* w_off;    /* n_atoms*n_proj */
    int n_lm;                  /* (max l + 1)^2 */
    const double* ylm_data;
    const long long* ylm_off;  /* n_atoms*n_lm */
    double gx, gy, gz;         /* Bloch vector (complex operator only) */
} qg_hamiltonian_desc;

/* ---- status / context -------------------------------------------------- */
const char* qg_status_string(int status);
/* Text of the last error the library recorded on this host thread's calls (empty if none). */
const char* qg_last_error(void);
int qg_version(void);

/* Creates a context on CUDA device `device` with its own non-blocking stream.
 * Replaces nothing in the reference (the reference has no device state). */
int qg_context_create(int device, qg_context* out);
/* Fails with QG_ERR_INVALID while operators built on the context are alive. */
int qg_context_destroy(qg_context ctx);
/* Work of this context is issued on `stream` (a cudaStream_t) from now on;
 * NULL selects the CUDA legacy default stream. A new context starts on its
 * own non-blocking stream. */
int qg_context_set_stream(qg_context ctx, void* stream);
/* Waits for the context's stream, then returns (and clears) the device status
 * word: QG_OK, or QG_ERR_TIMEOUT if a kernel's bounded wait gave up. */
int qg_context_synchronize(qg_context ctx);
/* Returns and clears the device status word without waiting for the stream. */
int qg_context_take_device_status(qg_context ctx);

/* ---- Hamiltonian ------------------------------------------------------- */
/* Builds the device operator: uploads V, compacts the cube tables into
 * sphere point lists (gather side) and a per-grid-point entry list (scatter
 * side). Replaces PseudoPotIntegrator::UpdatePosition (PseudoPotOperator.h:453)
 * plus the state QUMASUN_SINGLE/QUMASUN_MPI hold for mHamiltonianMatrix. */
int qg_hamiltonian_create(qg_context ctx, const qg_hamiltonian_desc* desc, qg_hamiltonian* out);
int qg_hamiltonian_destroy(qg_hamiltonian ham);
/* Changes the Bloch vector of an existing operator (k-point loop). */
int qg_hamiltonian_set_kvector(qg_hamiltonian ham, double gx, double gy, double gz);

/* HX[s] = H X[s] for ns states, DEVICE pointers, FP64.
 * Replaces ns calls of OpeA -> mHamiltonianMatrix(_ddm) (qumasun_single.matrix.h:19-40,
 * qumasun_mpi.matrix.h:20-43) and the bundled mHamiltonianMatrix_bundle_ddm (:46-104). */
int qg_hamiltonian_apply_d(qg_hamiltonian ham, int ns, const double* X, long long ldx,
                           double* HX, long long ldhx);
/* Same in FP32 (float states; V and projector tables rounded from FP64 once). */
int qg_hamiltonian_apply_f(qg_hamiltonian ham, int ns, const float* X, long long ldx,
                           float* HX, long long ldhx);
/* Same as qg_hamiltonian_apply_d with HOST buffers: copies X to the device,
 * applies H, copies HX back, and returns after HX is on the host. */
int qg_hamiltonian_apply_host_d(qg_hamiltonian ham, int ns, const double* X, double* HX);

/* Complex k-point operator H_k u = V u + V_NL(g) u - 1/2 (Lap + 2i g.grad - g^2) u
 * for ns split-complex states, DEVICE pointers, FP64: state s has its real part
 * at X + s*ldx and its imaginary part at X + s*ldx + N (ldx, ldhx >= 2N), the
 * reference's {re[N], im[N]} state layout (lobpcg_z_multi_mpi.h:1005-1012).
 * g is the operator's Bloch vector (descriptor or qg_hamiltonian_set_kvector);
 * the projectors carry exp(i g.r) at the unwrapped image position of each
 * cube point. FD order 8, 6 or 2 (KINETIC_8TH / _6TH / _2ND of qumasun_kpoint.matrix.h:78-86:
 * LaplasianKpoint8th/6th/2nd); order 4 returns QG_ERR_UNSUPPORTED (the reference has no
 * 4th-order k-point stencil).
 * Replaces OpeA(SoAComplex& Ax, const SoAComplex& x) of qumasun_kpoint.lobpcg.h:38-40
 * -> QUMASUN_KPOINT::mHamiltonianMatrix_ddm (qumasun_kpoint.matrix.h:25-50):
 * mPotentialMatrix_ddm on re and im, PseudoPotIntegrator_kpoint::ProjectionPP
 * (PseudoPotOperator_kpoint_v2.h:2581-2700), LaplasianKpoint8th_ddm
 * (GridDifferenceKpoint8th.h:325-368). */
int qg_hamiltonian_apply_z(qg_hamiltonian ham, int ns, const double* X, long long ldx,
                           double* HX, long long ldhx);
/* The k-point operator for nk k-points in one pass: kvecs = nk Bloch vectors (HOST,
 * 3 doubles each, bohr^-1), nsk states per k-point, state s of k-point k at
 * X + k*ldk + s*ldx (HX + k*ldkh + s*ldhx), DEVICE FP64, ldx/ldhx >= 2N,
 * ldk >= nsk*ldx. Each stencil work item and projector block carries its k-point's
 * coefficients and Bloch tables, so all k-points share one launch per phase. The
 * operator's own k-vector (qg_hamiltonian_set_kvector) is not used. No counterpart in
 * the reference, which loops over k (qumasun_kpoint.lobpcg.h:25-41). */
int qg_hamiltonian_apply_zk(qg_hamiltonian ham, int nk, const double* kvecs, int nsk, const double* X,
                            long long ldx, long long ldk, double* HX, long long ldhx, long long ldkh);
/* Complex64 states (FP32 {re[N], im[N]} per state): the same operator with FP32
 * stencil, potential, Bloch tables and projector sums (the FP32 counterpart of
 * qg_hamiltonian_apply_f for k-points); single k-vector / several k-points. */
int qg_hamiltonian_apply_zf(qg_hamiltonian ham, int ns, const float* X, long long ldx, float* HX, long long ldhx);
int qg_hamiltonian_apply_zkf(qg_hamiltonian ham, int nk, const double* kvecs, int nsk, const float* X,
                             long long ldx, long long ldk, float* HX, long long ldhx, long long ldkh);
/* qg_hamiltonian_apply_z with HOST buffers (ns * 2N doubles each, ldx = 2N). */
int qg_hamiltonian_apply_host_z(qg_hamiltonian ham, int ns, const double* X, double* HX);
/* qg_hamiltonian_apply_z with the phase timing of qg_hamiltonian_apply_timed_d. */
int qg_hamiltonian_apply_timed_z(qg_hamiltonian ham, int ns, const double* X, long long ldx,
                                 double* HX, long long ldhx, float* ms_phases);

/* qg_hamiltonian_apply_d with device-side phase timing (CUDA events on the
 * context stream; the call synchronizes): ms_phases[0] = projector
 * gather-contraction, [1] = stencil + local potential, [2] = nonlocal scatter
 * (the fused kernel reports its scatter inside [1]). Replaces the StopWatch
 * sectors 13 (PPNonlocal), 11 (K-operation) and 12 (V-operation) of
 * qumasun_mpi.matrix.h:29-41. */
int qg_hamiltonian_apply_timed_d(qg_hamiltonian ham, int ns, const double* X, long long ldx,
                                 double* HX, long long ldhx, float* ms_phases);
/* No counterpart in the reference (its CPU operator allocates freely).
 * Same result as qg_hamiltonian_apply_d (FP64, DEVICE pointers, context
 * stream), for callers that cannot call cudaMalloc at the point of the call:
 * hosts whose device memory belongs to another framework's allocator (a pool
 * that must not be bypassed), and time-critical loops that must not touch the
 * allocator. It allocates nothing: the projector coefficients go to a scratch
 * array compiled into the library, qg_noalloc_scratch_capacity() doubles
 * (4 MiB) per device that loads the library, held until the process exits,
 * which must hold ns16 * n_atoms * n_channels values (ns16 = ns rounded up to a
 * multiple of 16; n_channels = 4 for s+p projectors); larger batches return
 * QG_ERR_UNSUPPORTED before anything is launched. The first call on a device
 * looks up the array's device address (a CUDA runtime query, no allocation), so
 * make that first call before any stream capture. All calls on a device share
 * the array and it keeps the last call's contents: each call writes the slots
 * [0, ns) of every coefficient row before reading them; the padding slots
 * [ns, ns16) may be read but never reach HX. Calls that overlap on the GPU
 * (other streams, other threads) race and must be serialised by the caller. */
int qg_hamiltonian_apply_noalloc_d(qg_hamiltonian ham, int ns, const double* X, long long ldx,
                                   double* HX, long long ldhx);
/* Capacity, in doubles, of the fixed scratch array qg_hamiltonian_apply_noalloc_d uses. */
size_t qg_noalloc_scratch_capacity(void);

/* ---- LOBPCG ------------------------------------------------------------ */
typedef struct qg_lobpcg_options {
    int max_iter;       /* iteration limit (reference: iter_max) */
    double tol;         /* stop when max_j sum_i r_j(i)^2 dV < tol * dV (reference limit 1e-10,
                           lobpcg_d_multi.h:54, :525); <= 0 selects 1e-10 */
    int first_call;     /* 1: start with P = 0 and the 2n x 2n first step (reference is_first_time) */
    int precision;      /* QG_FP64: FP64 throughout; QG_MIXED_BF16X3: split-BF16x3 Gram products;
                           QG_FP32: FP32 Gram products (chunked, FP64 across chunks); both reduced
                           modes hand over to FP64 Gram products near convergence */
    int verbose;        /* 1: print (iteration, max residual) lines to stdout */
    int precond;        /* 0: none (the reference's solvers); 1: kinetic, w = (-1/2 Lap_FD + shift)^-1 r
                           applied in Fourier space with the FD stencil's own symbol; 2: kinetic
                           plus the learned correction of qg_hamiltonian_set_learned; 3: kinetic,
                           with the learned correction NN(r) as a fourth block of the
                           Rayleigh-Ritz basis [x, T r, NN(r), p] (real states, QG_FP64; one more
                           H application per iteration) */
    double precond_shift; /* shift (Ha) of the kinetic preconditioner; <= 0 selects 1.0 */
    int n_converge;     /* the lowest n_converge states must meet tol, the others are a guard
                           band against a degenerate multiplet at the cut; <= 0 or >= ns: all */
} qg_lobpcg_options;

typedef struct qg_lobpcg_report {
    int iterations;     /* LOBPCG iterations taken (H applications to R) */
    int converged;      /* 1 if the residual criterion was met */
    double max_residual;/* max_j sum_i r_j(i)^2 dV at exit */
    double ms_total;    /* device time of the solve */
    double ms_hamiltonian, ms_gram, ms_eigensolve, ms_rotate, ms_vector;  /* per-phase device time */
    int restarts;       /* iterations whose [x r p] Gram matrix was not positive definite at
                           working precision and that were solved on its numerically
                           nonsingular subspace (eigenvalues of B above 1e-12 max) */
    int mixed_iterations; /* QG_MIXED_BF16X3: iterations run with BF16x3 Gram products before
                           the hand-over to FP64 (residual below 1e-6 or stalled 3 iterations) */
} qg_lobpcg_report;

/* Block LOBPCG for the ns lowest eigenpairs of H, FP64 on the GPU.
 * Replaces EigenLOBPCG_d_multi (lobpcg_d_multi.h:23-545): same iteration (x
 * normalised with dV, residual r = Ax - (x.Ax dV) x, the 3n x 3n pencil
 * ([x r p]^T [Ax Ar Ap] dV, [x r p]^T [x r p] dV) -- 2n x 2n on the first step --
 * solved for its ns lowest pairs, P = R Cr + P Cp, X = X Cx + P, columns
 * renormalised, same stopping rule), with the Gram and rotation products as
 * DGEMMs (the w_dgemm path of lobpcg_d_multi_mpi.h:191-579) and the small
 * generalised eigenproblem solved on the GPU (replaces lapack_DSYGVX,
 * w_dsygvx.h:24-104). X (ns*N, in/out), P (ns*N, in/out, the reference's
 * "keep") and ev (ns, out) are HOST buffers, state-major. The pencil is
 * Jacobi-equilibrated (scaled to unit diag(B)) and solved with cuSOLVER's
 * sygvd; if B is still not positive definite, the step is solved on the span
 * of B's eigenvectors with eigenvalues above 1e-12 max (counted in
 * report->restarts) instead of stopping. A rotated Ritz vector whose |x|^2 dV drifts
 * from 1 by more than 1e-3 rolls the step back (the check of Eigen_d_multi_mpi,
 * lobpcg_d_multi_mpi.h:1305-1346): X and P are kept, the next step solves the [x r]
 * pencil from a full Gram (counted in report->restarts; 20 rollbacks end the solve with
 * QG_ERR_CHOLESKY). Returns QG_ERR_NOT_CONVERGED (results
 * still written) when max_iter is reached, QG_ERR_CHOLESKY if fewer than ns
 * independent directions remain. */
int qg_lobpcg_d(qg_hamiltonian ham, const qg_lobpcg_options* opt, int ns, double* ev, double* X,
                double* P, qg_lobpcg_report* report);
/* Same with DEVICE buffers X and P (ld = N); ev stays a host array. */
int qg_lobpcg_d_device(qg_hamiltonian ham, const qg_lobpcg_options* opt, int ns, double* ev,
                       double* X, double* P, qg_lobpcg_report* report);

/* Complex block LOBPCG for the k-point operator (qg_hamiltonian_apply_z) on ns
 * split-complex states: X and P are ns * 2N HOST doubles, state s = {re[N], im[N]}
 * at X + 2Ns. Same iteration, options, stopping rule (max_j |r_j|^2 dV < tol dV)
 * and statuses as qg_lobpcg_d; the Gram products are real DGEMMs over the re/im
 * columns combined into the Hermitian pencil S = (RR + II) + i (RI - IR), solved
 * in FP64 by cusolverDnZhegvd after Jacobi equilibration. The kinetic
 * preconditioner (precond = 1) applies the Gamma-point FD symbol to the real and
 * the imaginary part. Replaces LOBPCG::Eigen_z_multi_mpi (lobpcg_z_multi_mpi.h:988-1800:
 * MakeMatrix_z_blas :214-300, lapack_ZHEGVX w_zhegvx.h:24-107, NextVector_z :586-712)
 * as called by qumasun_kpoint.lobpcg.h:32-41. */
int qg_lobpcg_z(qg_hamiltonian ham, const qg_lobpcg_options* opt, int ns, double* ev, double* X,
                double* P, qg_lobpcg_report* report);
/* Complex LOBPCG for nk k-points in one solve (the batched form of running
 * qg_lobpcg_z once per k-point): kvecs = nk Bloch vectors (HOST, 3 each), nsk states
 * per k-point, X and P DEVICE, [k][s] state-major ({re[N], im[N]} per state), ev HOST
 * (nk * nsk). H, norms, residuals and the preconditioner run over all k-points' states in
 * single launches; Gram products are DGEMMs per k-point, rotations strided-batched DGEMMs
 * over k; the nsk-state pencils are solved k-point by k-point, and a k-point whose states
 * have converged is frozen (no further rotation or solve). FP64; precond 0 or 1; stops when the
 * lowest n_converge states of every k-point meet tol. The report carries iterations,
 * convergence, max_residual, ms_total and restarts. No counterpart in the reference,
 * which loops over k-points (qumasun_kpoint.lobpcg.h:25-41). */
int qg_lobpcg_zk_device(qg_hamiltonian ham, const qg_lobpcg_options* opt, int nk, const double* kvecs, int nsk,
                        double* ev, double* X, double* P, qg_lobpcg_report* report);
/* Same with DEVICE buffers X and P (ld = 2N); ev stays a host array. */
int qg_lobpcg_z_device(qg_hamiltonian ham, const qg_lobpcg_options* opt, int ns, double* ev,
                       double* X, double* P, qg_lobpcg_report* report);
/* Real LOBPCG (qg_lobpcg_d_device) on several independent cells at once: cell c has
 * operator hams[c], options opts[c], ns[c] states, DEVICE X[c] / P[c] (P may be NULL
 * when every opts[c].first_call is set), HOST ev[c]; reports[c] and status[c] (either
 * may be NULL) receive each cell's report and status. Each cell must use its own
 * context (its stream and library handles); the cells' solves run concurrently on
 * their streams, so small cells fill the GPU together. Returns QG_OK or the first
 * failing cell's status. No counterpart in the reference, which solves one cell per
 * run (EigenLOBPCG_d_multi, lobpcg_d_multi.h:23-27, called per spin by
 * qumasun_single.lobpcg.h:17-34). */
int qg_lobpcg_cells_device(int ncells, const qg_hamiltonian* hams, const qg_lobpcg_options* opts, const int* ns,
                           double* const* ev, double* const* X, double* const* P, qg_lobpcg_report* reports,
                           int* status);

/* No counterpart in the reference (its Gram products are FP64 BLAS, w_dgemm.h:32-36).
 * C (m x m, column-major, ld m) = alpha * A^T B for DEVICE blocks A, B (N x m,
 * ld N; B NULL means B = A) through the mixed-precision Gram of QG_MIXED_BF16X3:
 * pieces = 2 or 3 bf16 pieces per value on the library's tcgen05 kernel (FP32
 * accumulation over one 64-row K block, FP64 across blocks; N a multiple of 8),
 * pieces = 0 the cuBLAS BF16 hi/lo path (FP32 over 1024-row chunks), pieces = -1
 * FP32 copies and FP32 GEMMs over the same chunks (the Gram of QG_FP32), pieces = 7
 * the FP64-accurate int8 slice products of QG_FP64_INT8. Waits for the stream; returns
 * QG_ERR_UNSUPPORTED if the tensor-core path cannot take N. */
int qg_gram_mixed_d(qg_context ctx, long long N, int m, const double* A, const double* B, double alpha,
                    double* C, int pieces);

/* The Gram product the real LOBPCG uses for pencils of up to 128 columns
 * (MakeMatrix_d_blas, lobpcg_d_multi_mpi.h:191-250, with K = the grid): C (ma x mb,
 * column-major, ld ma) = alpha * A^T B for DEVICE blocks A (N x ma) and B (N x mb),
 * ld N, with K split over the GPU and the partial sums added in a fixed order. Any
 * ma, mb (64 x 64 output tiles); waits for the stream. */
int qg_gram_small_d(qg_context ctx, long long N, int ma, int mb, const double* A, const double* B, double alpha,
                    double* C);

/* ---- learned preconditioner ------------------------------------------------
 * No counterpart in the reference (its solvers are unpreconditioned). A 4-layer
 * periodic 3D convolutional network (3^3 kernels, channels 2 -> 16 -> 16 -> 16 -> 1,
 * ReLU after the first three, BF16 weights and activations, FP32 accumulation):
 *   NN(r) = rms(r) * net([r / rms(r), V / vscale]),  rms(r) = sqrt(mean r^2),
 * used by LOBPCG (precond = 2) as w = T r + NN(r), T the kinetic preconditioner.
 * Parameters: qg_learned_num_params() floats, per layer the weights [cout][cin][27]
 * (taps x fastest) followed by the cout biases. A new network has all parameters
 * zero (NN = 0). The handle counts as an operator of its context. */
int qg_learned_num_params(void);
int qg_learned_create(qg_context ctx, qg_learned* out);
int qg_learned_destroy(qg_learned nn);
int qg_learned_set_params(qg_learned nn, const float* params, int n);  /* HOST params */
int qg_learned_get_params(qg_learned nn, float* params, int n);
/* The four layers of the forward pass run on the tensor cores (tcgen05.mma kind::f16,
 * BF16 operands, FP32 accumulation in TMEM; one 16 x 16 channel MMA per 3^3 tap over
 * halo planes staged in shared memory) when nx is a multiple of 8 -- the default;
 * on = 0 selects the CUDA-core kernels (the two differ only in the order of the FP32
 * sums). The backward pass always runs on the CUDA-core kernels. Waits for the stream. */
int qg_learned_set_tensor_cores(qg_learned nn, int on);
/* out[s] (+)= NN(R[s]) for ns states on an nx x ny x nz grid; R, V, out DEVICE FP64. */
int qg_learned_apply_d(qg_learned nn, int nx, int ny, int nz, int ns, const double* R, long long ldr,
                       const double* V, double vscale, double* out, long long ldo, int accumulate);
/* Loss sum_s |net_s - Y[s]/rms(R[s])|^2 / sum_s |Y[s]/rms(R[s])|^2 of a batch (Y: the wanted
 * NN(R) in the units of R, DEVICE FP64) and its gradient (grad_host: HOST, num_params
 * floats, may be NULL); waits for the stream. */
int qg_learned_gradient(qg_learned nn, int nx, int ny, int nz, int ns, const double* R, long long ldr,
                        const double* V, double vscale, const double* Y, long long ldy, double* loss,
                        float* grad_host);
/* qg_learned_gradient followed by one Adam step (beta 0.9 / 0.999) with learning rate lr. */
int qg_learned_train_step(qg_learned nn, int nx, int ny, int nz, int ns, const double* R, long long ldr,
                          const double* V, double vscale, const double* Y, long long ldy, float lr,
                          double* loss);
/* R[s] <- T R[s] in place, T = (-1/2 Lap_FD + shift)^-1 the kinetic preconditioner of
 * LOBPCG's precond = 1 (DEVICE R, ns states, ldr = N). */
int qg_hamiltonian_precondition_d(qg_hamiltonian ham, int ns, double* R, long long ldr, double shift);
/* Attaches a network to an operator for LOBPCG's precond = 2 (NULL detaches). */
int qg_hamiltonian_set_learned(qg_hamiltonian ham, qg_learned nn, double vscale);

/* Batched small generalised eigensolver, FP64, DEVICE pointers, context stream:
 * for b < batch, A_b z = lambda B_b z with A_b = A + b*stride, B_b = B + b*stride
 * (k x k, column-major, leading dimension lda, lower triangles read), all k
 * eigenpairs ascending into w + b*k and Z + b*k*k (column-major, ld k).
 * Replaces lapack_DSYGVX (w_dsygvx.h:24-104: ITYPE 1, JOBZ V, RANGE A) for
 * k <= 80; larger k returns QG_ERR_UNSUPPORTED. info (host, batch ints, may be
 * NULL) receives 0, or 1 where B_b is not positive definite; the call waits
 * for the stream when info is given. */
int qg_sygv_small_batched_d(qg_context ctx, int batch, int k, const double* A, const double* B, int lda,
                            long long stride, double* w, double* Z, int* info);
/* Complex Hermitian counterpart: A, B, Z hold interleaved {re, im} doubles (k x k
 * complex, column-major, leading dimension lda complex elements, stride in complex
 * elements, lower triangles read); Z + b*k*k (ld k). Replaces lapack_ZHEGVX
 * (w_zhegvx.h:24-107: ITYPE 1, JOBZ V, RANGE A) for k <= 56, the pencils of the
 * k-point LOBPCG with up to 18 states per k-point. info as above. */
int qg_hegv_small_batched_z(qg_context ctx, int batch, int k, const double* A, const double* B, int lda,
                            long long stride, double* w, double* Z, int* info);

/* Selects the stencil kernel of an operator's real-state apply: 0 = the engine's
 * choice (default: the TMA ring kernel with two grid rows per thread where the shape
 * and alignment allow -- V through the ring in FP64, from global memory in FP32 -- else
 * the other ring kernels, else the register-window kernel),
 * 1 = always the register-window kernel (any shape), 2 = the one-plane ring
 * kernel, 3 = the two-plane ring kernel, 4 = the ring kernel with two grid rows per
 * thread and V streamed through the ring, 5 = the same with V read one plane ahead from
 * global memory (2-5 fall back as 0 does where the shape does not fit). All give the same bits. Complex states use the one-plane ring kernel
 * unless 1 is set. */
int qg_hamiltonian_set_stencil_kernel(qg_hamiltonian ham, int variant);
/* Tuning of the nonlocal passes: states per projection block (1, 2, 4, 8 or 16;
 * complex states use at most 4), states per scatter group of the real apply (4 or
 * 8), and blocks per atom in the projection (1-8, one thread-block cluster; the
 * engine's choice follows the cell alone: 1 for cells of more than 16 atoms, else
 * one per 4096 sphere points of the largest atom); 0 = the
 * engine's choice. The block sizes do not change the result (same sums in the same
 * order); the parts per atom change the summation order of the projections (last
 * bits only), and the engine's choice never depends on the number of states. */
int qg_hamiltonian_set_nonlocal_blocking(qg_hamiltonian ham, int project_states, int scatter_states,
                                         int project_parts);
/* Real-state LOBPCG (qg_lobpcg_d, _device, cells) with more than 128 Gram columns: 1
 * (default) forms the steady-state pencil from the previous rotation -- only the blocks
 * with the new residuals are tall products ([x r p]^T A r, [x r p]^T r), the x/p blocks
 * are Z^T S Z of the last pencil (the direct update of NextMatrix_d,
 * lobpcg_d_multi_mpi.h:264-460) -- with a full Gram every 10 iterations and after any
 * 2n step, rank-revealing solve or rollback; 0 forms the full Gram every iteration. */
int qg_hamiltonian_set_gram_reuse(qg_hamiltonian ham, int on);
/* Test hook of the bounded waits: with on = 1 the producer lane of the ring stencil
 * kernels (real states) issues no copy, so every consumer's bounded mbarrier wait
 * (about 2^31 SM clocks) runs out; the kernels then wind down, record QG_ERR_TIMEOUT
 * in the context's device status word (qg_context_synchronize /
 * qg_context_take_device_status) and the context stays usable. 0 restores normal
 * operation. Nothing in the library sets it. */
int qg_hamiltonian_test_stall(qg_hamiltonian ham, int on);
/* Autotuner of the real-state apply (no counterpart in the reference): times, on the
 * caller's DEVICE block of ns states (X in, HX overwritten), the launch shapes that leave
 * every bit of H|psi> unchanged -- stencil kernel (variants 2-5 of
 * qg_hamiltonian_set_stencil_kernel), states per projection block (2, 4, 8, 16) and per
 * scatter group (4, 8) -- one dimension at a time (the phases are independent), best of
 * three CUDA-event timed applies each, and keeps the fastest in the operator.
 * choice (3 ints, may be NULL) receives {stencil variant, projection states, scatter
 * states}; ms_phases (3 floats, may be NULL) the chosen configuration's projection,
 * stencil + V and scatter times. The projector split over blocks is left to the cell
 * rule: it changes the summation order. About 40 applies. */
int qg_hamiltonian_autotune_d(qg_hamiltonian ham, int ns, const double* X, long long ldx, double* HX,
                              long long ldhx, int* choice, float* ms_phases);
int qg_hamiltonian_autotune_f(qg_hamiltonian ham, int ns, const float* X, long long ldx, float* HX,
                              long long ldhx, int* choice, float* ms_phases);
/* Number of kernel launches one apply of `ns` states issues (for launch accounting). */
int qg_hamiltonian_launches_per_apply(qg_hamiltonian ham, int ns);

/* ---- SCF-step neighbours of the eigensolver ---------------------------- */

/* rho[i] (+)= sum_s occ[s] * psi_s[i]^2 over the states with occ[s] > 0, in state
 * order, each term rounded as the reference forms it ((psi*psi)*occ added to rho, no
 * fused multiply-add): the sums equal the reference's bit for bit on the same inputs.
 * X: ns real states on the DEVICE, state s at X + s*ldx (ldx >= N); occ: HOST, ns
 * values; rho: DEVICE, N values, zeroed first unless accumulate != 0. Context stream;
 * returns after the kernel has run. Replaces QUMASUN_SINGLE::mSetDensityOne
 * (qumasun_single.density.h:10-27). */
int qg_density_d(qg_context ctx, long long N, int ns, const double* X, long long ldx, const double* occ,
                 double* rho, int accumulate);
/* Complex {re[N], im[N]} states (ldx >= 2N): rho += occ * (re^2 + im^2). Replaces
 * QUMASUN_KPOINT::mSetDensityOne (qumasun_kpoint.density.h:11-33). */
int qg_density_z(qg_context ctx, long long N, int ns, const double* X, long long ldx, const double* occ,
                 double* rho, int accumulate);
/* Fermi occupations (2 electrons per state) of n eigenvalues (HOST, ascending) for
 * n_electrons electrons at temperature kbT (Ha): bisection on the chemical potential
 * from [ev[0], 16 |ev[n-1]|-ish] down to 1e-9 Ha, occ[s] = 2/(exp(min((ev-mu)/kbT, 80))+1).
 * HOST arithmetic (a few hundred exponentials per step). Replaces
 * QUMASUN_SINGLE::mSetOccupancySpinOff (qumasun_single.occupancy.h:19-55) with
 * SetOccupancy (SetOccupancy.h:7-18). */
int qg_occupancy(double kbT, int n, const double* ev, int n_electrons, double* occ, double* mu);
/* Spin-polarised form: one state per electron in each spin channel, one shared mu.
 * Replaces mSetOccupancySpinOn (qumasun_single.occupancy.h:62-109). */
int qg_occupancy_spin(double kbT, int n, const double* ev_up, const double* ev_dn, int n_electrons,
                      double* occ_up, double* occ_dn, double* mu);

typedef struct qg_poisson_s* qg_poisson;
/* FFT Poisson + LDA potential builder for an nx x ny x nz periodic grid of spacing
 * (hx, hy, hz): owns a cuFFT plan and an N-point complex buffer on the context's device.
 * The context must outlive it. */
int qg_poisson_create(qg_context ctx, int nx, int ny, int nz, double hx, double hy, double hz, qg_poisson* out);
int qg_poisson_destroy(qg_poisson p);
/* V_tot = V_ext + V_hart + V_x + V_c on the DEVICE (context stream), all arrays of N
 * doubles: V_hart from the periodic Poisson equation solved by FFT, 4 pi/|k|^2 on the
 * folded wave numbers with the k = 0 term dropped, inverse transform scaled by 1/N;
 * V_x, V_c the Perdew-Zunger 1981 LDA potentials of rho + pcc (zero below 1e-8).
 * pcc may be NULL (no core charge); vhart, vx, vc may be NULL (not returned).
 * Replaces QUMASUN_SINGLE::mSetPotential for KohnSham_PP without spin
 * (qumasun_single.potential.h:33-43): mSetPotentialVhart (:101-200, the same solve as
 * SetPotentialByPoissonFFT, poisson_fft.h:14-128) and mSetPotentialVxc (:311-317,
 * Calc_XC_LDA, Vxc.h:41-70). */
int qg_potential_lda_d(qg_poisson p, const double* rho, const double* pcc, const double* vext, double* vtot,
                       double* vhart, double* vx, double* vc);

/* One fourth-order Taylor step psi <- sum_{j=0..4} (-i dt H)^j / j! psi of ns complex
 * {re[N], im[N]} states (DEVICE, in place, ldx >= 2N) under the operator at its
 * k-vector (FD order 2, 6 or 8): four applications of H to the whole block, each followed by
 * the update of that order. Work: two blocks of ns states kept by the operator.
 * Replaces QUMASUN::TimeEvoH4 (qumasun_td.time_evo_H4.h:13-60), which steps one state
 * at a time. */
int qg_td_taylor4_z(qg_hamiltonian ham, int ns, double dt, double* X, long long ldx);

/* Nonlocal energy and forces of ns real states (DEVICE X, state s at X + s*ldx): for
 * every state, inner = dV <p|psi> over all projector channels and e_state[s] =
 * sum E inner^2 (EnergyPPnonlocal, PseudoPotOperator.h:775-816); for the states with
 * occ[s] > 0, dpsi = -2 occ grad psi (8th-order FD gradient, Gradient8th,
 * GridGradient8th.h:19-235), dinner = dV <p|dpsi> and forces[3a + d] +=
 * sum E inner dinner_d; *ev_sum = sum occ[s] e_state[s]. occ, forces (3 per atom,
 * accumulated), e_state (may be NULL) and ev_sum (may be NULL) are HOST. Replaces
 * QUMASUN_MPI::mGetForcePseudoNonlocal (qumasun_mpi.force.h:227-254) with
 * PseudoPotIntegrator_mpi::ForceNonlocal (PseudoPotOperator_mpi_v2.h:905-1010). */
int qg_nonlocal_force_d(qg_hamiltonian ham, int ns, const double* X, long long ldx, const double* occ,
                        double* forces, double* e_state, double* ev_sum);

#ifdef __cplusplus
}
#endif
#endif /* QUMASUN_B200_H */
