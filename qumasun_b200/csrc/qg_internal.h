// Internal declarations shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <vector>

#include "../../include/qumasun_b200.h"

#define QG_CUDA_TRY(expr)                                                       \
    do {                                                                        \
        cudaError_t qg_e_ = (expr);                                             \
        if (qg_e_ != cudaSuccess) {                                             \
            qg_set_last_error(#expr, cudaGetErrorString(qg_e_), __FILE__, __LINE__); \
            return qg_e_ == cudaErrorMemoryAllocation ? QG_ERR_NOMEM : QG_ERR_CUDA; \
        }                                                                       \
    } while (0)

#define QG_TRY(expr)                    \
    do {                                \
        int qg_s_ = (expr);             \
        if (qg_s_ != QG_OK) return qg_s_; \
    } while (0)

void qg_set_last_error(const char* what, const char* msg, const char* file, int line);

// A device buffer that only grows.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t want) {
        if (want <= bytes) return QG_OK;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        if (cudaMalloc(&ptr, want) != cudaSuccess) return QG_ERR_NOMEM;
        bytes = want;
        return QG_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

struct qg_context_s {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    void* blas = nullptr;      // cublasHandle_t, created on first use
    void* solver = nullptr;    // cusolverDnHandle_t, created on first use
    int live_hamiltonians = 0; // the context outlives every operator built on it
    int* dev_status = nullptr; // device status word set by kernels whose bounded waits gave up
    void* gram_cache = nullptr; // qg::MixedGram buffers kept by qg_gram_mixed_d across calls
    DevBuf small;               // per-call state lists of the density entry points
};

// Frees the context's qg_gram_mixed_d buffers (gram_mixed.cu).
void qg_release_gram_cache(qg_context c);

// Nonlocal projector tables on the device, in two orders:
//  gather side (atom-major): atom a owns points [atom_off[a], atom_off[a+1]) of
//    pt_g (grid index) and tab[ch*npts + p] (channel values w*Y);
//  scatter side (grid-point-major): grid point g owns entries
//    [row[g], row[g+1]) with the atom id ent_atom[e] and channel values
//    ent_val[e*nch + ch].
struct DevProjectors {
    int na = 0, nch = 0;
    long long npts = 0, nent = 0;
    long long max_atom_pts = 0;  // sphere points of the largest atom
    int* atom_off = nullptr;
    int* pt_g = nullptr;
    double* tab_d = nullptr;
    float* tab_f = nullptr;
    double* ch_scale = nullptr;  // E_k * dV per (atom, channel)
    double* ch_dv = nullptr;     // dV per (atom, channel) with a projector (0 for padding channels)
    double* ch_E = nullptr;      // E_k per (atom, channel) (0 for padding channels)
    int* row = nullptr;
    int* ent_atom = nullptr;
    double* ent_val_d = nullptr;
    float* ent_val_f = nullptr;
    // k-point (complex) side: unwrapped grid coordinates of each point (3 per
    // point, the image the cube point came from), the point of each scatter
    // entry, and the Bloch-phase tables for the k-vector zg:
    //   ztab[ch*npts + p] = tab * cos(theta_p), ztab[(nch + ch)*npts + p] = tab * sin(theta_p),
    //   zent[(e*nch + ch)*2 + {0,1}] = ent_val * (cos, sin)(theta_p(e)),
    // theta_p = g . (h * u_p)
    int* pt_u = nullptr;
    int* ent_pt = nullptr;
    double* ztab = nullptr;
    double* zent = nullptr;
    std::vector<double> zk;  // k-vectors (3 per k-point) the tables were built for
    int zcap = 0;            // k-points the table buffers hold
    bool zready = false;
    // the same tables in FP32 for complex64 states
    float* ztab_f = nullptr;
    float* zent_f = nullptr;
    std::vector<double> zk_f;
    int zcap_f = 0;
    bool zready_f = false;
};

namespace qg {
struct KineticPrecond;
}

struct qg_hamiltonian_s {
    qg_context ctx = nullptr;
    int nx = 0, ny = 0, nz = 0;
    double hx = 0, hy = 0, hz = 0;
    int order = 8;
    double gx = 0, gy = 0, gz = 0;
    double* V_d = nullptr;
    float* V_f = nullptr;
    DevProjectors pj;
    DevBuf coef;      // projector coefficients E*dV*<p|psi>, [ns][na*nch]
    DevBuf xio, hxio; // staging for the host-buffer entry point
    DevBuf kco;       // per-k-point stencil coefficients of a multi-k apply
    DevBuf scf_work;  // propagation blocks, gradients and inner products (scf.cu)
    cudaStream_t io_in = nullptr, io_out = nullptr;  // copy streams of the host-buffer entry points
    int ty = 1;       // grid rows per stencil tile
    // stencil kernel of the real-state apply: 0 = engine's choice, 1 = register-window
    // kernel (any shape), 2 = one-plane TMA ring, 3 = two-plane TMA ring, 4 = two rows per
    // thread with V in the ring
    int stencil_variant = 0;
    int proj_sb = 0;     // states per projection block (0: chosen per launch)
    int proj_parts = 0;  // blocks (one cluster) per atom in the projection (0: from the cell)
    int scatter_sg = 0;  // states per scatter group (0: 8)
    int test_stall = 0;  // test hook: ring-stencil producers issue nothing (bounded waits run out)
    int gram_reuse = 1;  // LOBPCG: steady-state Gram pencil from the last rotation (0: full Gram every step)
    qg::KineticPrecond* precond = nullptr;  // LOBPCG preconditioner, built on first use
    qg_learned learned = nullptr;           // network of precond = 2 (qg_hamiltonian_set_learned)
    double learned_vscale = 1.0;
    long long N() const { return (long long)nx * ny * nz; }
};

namespace qg {

// Stencil tile geometry: ty grid rows of full x-rows per thread block.
int pick_tile_rows(int nx, int ny);
int stencil_radius(int order);

// Launchers (hamiltonian.cu).
// Device-time accounting by phase: mark(tag) records an event; the time up to
// the next mark is charged to `tag` (0 projection, 1 stencil + V, 2 scatter).
struct PhaseTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> tag;
    void mark(int t, cudaStream_t st) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev.push_back(e);
        tag.push_back(t);
    }
    void totals(float* ms3) {
        ms3[0] = ms3[1] = ms3[2] = 0.f;
        if (!ev.empty()) cudaEventSynchronize(ev.back());
        for (size_t i = 0; i + 1 < ev.size(); ++i) {
            float d = 0.f;
            cudaEventElapsedTime(&d, ev[i], ev[i + 1]);
            if (tag[i] >= 0 && tag[i] < 3) ms3[tag[i]] += d;
        }
    }
    ~PhaseTimer() {
        for (auto e : ev) cudaEventDestroy(e);
    }
};

// Host-buffer apply, pipelined over kHostChunks chunks of states through the
// staging buffers h->xio / h->hxio (hamiltonian.cu). Each state is `row` doubles;
// apply(nc, x_dev, hx_dev) queues the operator on the context stream.
constexpr int kHostChunks = 8;
int host_pipelined_apply(qg_hamiltonian h, int ns, long long row, const double* X, double* HX,
                         const std::function<int(int, const double*, double*)>& apply);

// Opts a kernel in to the device's largest dynamic shared memory (the opt-in maximum
// less the kernel's static shared memory). Every launcher sets this same value, so
// host threads that launch one kernel with different shared-memory sizes at once (the
// concurrent cell solves) never lower the limit under each other's launches.
template <typename K>
inline cudaError_t allow_max_dynamic_smem(K* kern) {
    int dev = 0, mx = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kern));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(kern), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                mx - (int)fa.sharedSizeBytes);
}

// Launch with `cluster_x` blocks per thread-block cluster along x (1: no cluster).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_clustered(void (*kern)(KArgs...), dim3 grid, dim3 block, int cluster_x, size_t smem,
                                    cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster_x;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = cluster_x > 1 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Blocks per atom of the projection (or the forced value), from the cell alone so that
// results never depend on the batch: one block per atom for cells of more than 16
// atoms (enough blocks already), and for smaller cells (solved with few states, where
// each block's serial walk over its points sets the time) one per kProjPartPoints
// sphere points of the largest atom, at most 8 (the portable cluster size). Measured on
// 8-, 64- and 216-atom diamond cells at 16-256 real and 16-128 complex states; on the
// large cells 2 parts were within 2 % of 1. Two parts per atom with every block walking
// all state groups in turn (so that all atoms sweep the groups together and the sphere
// overlaps hit L2) measured slower on the 64-atom cell, 0.69 against 0.49 ms at 256
// states: 128 blocks hide less gather latency than 2048 (atom, group) blocks.
constexpr int kProjPartPoints = 4096;
inline int project_parts(const DevProjectors& pj, int forced) {
    if (forced > 0) return forced;
    if (pj.na > 16) return 1;
    const long long p = std::max<long long>(1, (pj.max_atom_pts + kProjPartPoints - 1) / kProjPartPoints);
    return (int)std::min<long long>(8, p);
}

// Row length of the channel-major projector coefficients [na * nch][ld]: the state
// count rounded up to 16, so every row starts 128-byte aligned and the scatter's
// 16-byte loads of a state group never leave the row.
inline long long coef_ld(int ns) { return (ns + 15) / 16 * 16; }

// Elements of projector-coefficient scratch ([n_atoms * n_channels][coef_ld(ns)]) one apply of ns states needs.
size_t coef_scratch_elems(qg_hamiltonian h, int ns);
// Doubles of complex coefficient scratch ([nk][n_atoms * n_channels][coef_ld(nsk)] {re, im})
// one k-point apply of nk k-points x nsk states needs.
size_t coef_scratch_elems_z(qg_hamiltonian h, int nk, int nsk);

template <typename T>
int apply_hamiltonian(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx,
                      T* coef_scratch, cudaStream_t st, PhaseTimer* pt = nullptr);

// Inner products dV <p_{a,ch}|psi_s> of ns real states, channel-major like the
// operator's coefficients: coef[(a * nch + ch) * ldc + s] (hamiltonian.cu).
int project_inner_d(qg_hamiltonian h, int ns, const double* X, long long ldx, double* coef, long long ldc,
                    cudaStream_t st);

// Complex k-point H (kpoint.cu): state s has its real part at X + s*ldx and its
// imaginary part N elements later; coef_scratch holds 2*coef_scratch_elems(h, ns) doubles.
template <typename T>
int apply_hamiltonian_z(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx,
                        T* coef_scratch, cudaStream_t st, PhaseTimer* pt = nullptr);
// Several k-points in one pass: nk k-vectors kv (3 each, bohr^-1), nsk states per k-point,
// state s of k-point k at X + k*ldk + s*ldx (HX + k*ldkh + s*ldhx); coef_scratch holds
// 2*coef_scratch_elems(h, nk*nsk) doubles.
template <typename T>
int apply_hamiltonian_zk(qg_hamiltonian h, int nk, const double* kv, int nsk, const T* X, long long ldx,
                         long long ldk, T* HX, long long ldhx, long long ldkh, T* coef_scratch, cudaStream_t st,
                         PhaseTimer* pt = nullptr);

}  // namespace qg
