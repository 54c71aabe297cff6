// Kohn-Sham H|psi> on the device (mHamiltonianMatrix_ddm, qumasun_mpi.matrix.h:20-43):
//   H psi = V psi + sum_atoms sum_k E_k sum_m |p_km> dV <p_km|psi> - 1/2 Lap psi.
//
// Main path (shapes the TMA kernel accepts), three launches for a block of states:
//   k_project     c[a,ch][s] = E_ch dV sum_{p in sphere(a)} tab[ch][p] psi_s[g(p)]
//                 (InnerProd_1S_1R / InnerProd_2S_1R of ProjectionPP, PseudoPotOperator.h:740-772,
//                 all atoms, channels and states at once);
//   k_stencil_tma H psi = V psi - 1/2 Lap psi (stencil_tma.cu: persistent, TMA-staged);
//   k_scatter_all H psi[s][g] += sum_{entries e of g} sum_ch val[e][ch] c[a_e,ch][s]
//                 (Add_1S / Add_2S of ProjectionPP turned into a per-point gather, no atomics).
// Fallback path (any shape): k_project, then k_hamiltonian, a register-window
// stencil kernel with the per-point scatter fused in.
//
// k_hamiltonian data flow (per thread block: SPB states, ty full x-rows, a slab of z):
// the block marches up z; each thread keeps its own column's 2R+1 z-values in
// registers, stages the current plane (ty rows + R halo rows above and below,
// and R wrapped columns left and right) in shared memory for the x/y
// neighbours, and prefetches the plane R+1 ahead while it computes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <vector>

#include <cooperative_groups.h>

#include "qg_internal.h"
#include "stencil_common.cuh"
#include "precond.h"

namespace cg = cooperative_groups;

namespace qg {

int stencil_radius(int order) {
    switch (order) {
        case 2: return 1;
        case 4: return 3;
        case 6: return 3;
        case 8: return 4;
        default: return -1;
    }
}

int pick_tile_rows(int nx, int ny) {
    int best = 0;
    for (int t = 1; t <= 16; ++t)
        if (ny % t == 0 && nx * t <= 1024) best = t;
    return best;
}

// Laplacian at one point. p points at the centre in the staged plane (row pitch W);
// q holds the centre's column z-values q[R-R..R+R].
template <typename T, int ORDER, int R>
__device__ __forceinline__ T stencil_point(const T* __restrict__ p, int W, const T* q,
                                           const HamArgs<T>& a) {
    const T c = q[R];
    if constexpr (ORDER == 2) {
        // Laplasian2nd_halo_f (GridDifference2nd.h:1027-1031)
        return a.cx[0] * (p[1] + p[-1] - T(2) * c) + a.cy[0] * (p[W] + p[-W] - T(2) * c) +
               a.cz[0] * (q[R + 1] + q[R - 1] - T(2) * c);
    } else if constexpr (ORDER == 4) {
        // Laplasian4th_halo_f (GridDifference4th.h:528-530), composed 7-point stencil
        return a.cx[2] * ((p[3] + p[-3]) - T(54) * (p[2] + p[-2]) + T(783) * (p[1] + p[-1]) - T(1460) * c) +
               a.cy[2] * ((p[3 * W] + p[-3 * W]) - T(54) * (p[2 * W] + p[-2 * W]) +
                          T(783) * (p[W] + p[-W]) - T(1460) * c) +
               a.cz[2] * ((q[R + 3] + q[R - 3]) - T(54) * (q[R + 2] + q[R - 2]) +
                          T(783) * (q[R + 1] + q[R - 1]) - T(1460) * c);
    } else if constexpr (ORDER == 6) {
        // Laplasian6th_halo_f (GridDifference6th.h:425-429)
        T d = a.c0 * c;
        d += a.cx[2] * (p[3] + p[-3]) + a.cx[1] * (p[2] + p[-2]) + a.cx[0] * (p[1] + p[-1]);
        d += a.cy[2] * (p[3 * W] + p[-3 * W]) + a.cy[1] * (p[2 * W] + p[-2 * W]) + a.cy[0] * (p[W] + p[-W]);
        d += a.cz[2] * (q[R + 3] + q[R - 3]) + a.cz[1] * (q[R + 2] + q[R - 2]) + a.cz[0] * (q[R + 1] + q[R - 1]);
        return d;
    } else {
        // Laplasian8th_halo_f (GridDifference8th.h:141-145)
        T d = a.c0 * c;
        d += a.cx[3] * (p[4] + p[-4]) + a.cx[2] * (p[3] + p[-3]) + a.cx[1] * (p[2] + p[-2]) + a.cx[0] * (p[1] + p[-1]);
        d += a.cy[3] * (p[4 * W] + p[-4 * W]) + a.cy[2] * (p[3 * W] + p[-3 * W]) +
             a.cy[1] * (p[2 * W] + p[-2 * W]) + a.cy[0] * (p[W] + p[-W]);
        d += a.cz[3] * (q[R + 4] + q[R - 4]) + a.cz[2] * (q[R + 3] + q[R - 3]) +
             a.cz[1] * (q[R + 2] + q[R - 2]) + a.cz[0] * (q[R + 1] + q[R - 1]);
        return d;
    }
}

// One thread block: states [s0, s0+SPB), grid rows [y0, y0+ty), planes [zs, ze).
// blockDim.x == nx*ty (each thread owns one (ix, iy) column).
template <typename T, int ORDER, int SPB>
__global__ void __launch_bounds__(1024) k_hamiltonian(const HamArgs<T> a) {
    constexpr int R = ORDER == 2 ? 1 : (ORDER == 8 ? 4 : 3);
    constexpr int Q = 2 * R + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);

    const int nx = a.nx, ny = a.ny, nz = a.nz, ty = a.ty;
    const int W = nx + 2 * R;
    const int rows = ty + 2 * R;
    const int t = threadIdx.x;
    const int ix = t % nx;
    const int ly = t / nx;
    const int y0 = blockIdx.x * ty;
    const int iy = y0 + ly;
    const int s0 = blockIdx.y * SPB;
    const int zs = blockIdx.z * a.zslab;
    const int ze = min(nz, zs + a.zslab);
    if (zs >= ze) return;
    const long long plane = (long long)nx * ny;
    const long long col = (long long)iy * nx + ix;

    const T* Xs[SPB];
    bool valid[SPB];
#pragma unroll
    for (int s = 0; s < SPB; ++s) {
        valid[s] = (s0 + s) < a.ns;
        Xs[s] = a.X + (long long)(valid[s] ? s0 + s : s0) * a.ldx;
    }

    T q[SPB][Q];
#pragma unroll
    for (int s = 0; s < SPB; ++s)
#pragma unroll
        for (int d = 0; d < Q; ++d) q[s][d] = Xs[s][wrap_idx(zs - R + d, nz) * plane + col];

    for (int z = zs; z < ze; ++z) {
        // prefetch the plane entering the register window next step
        T nq[SPB];
        const bool more = (z + 1) < ze;
        if (more) {
            const long long off = (long long)wrap_idx(z + R + 1, nz) * plane + col;
#pragma unroll
            for (int s = 0; s < SPB; ++s) nq[s] = Xs[s][off];
        }
        // stage this plane's interior value (and its wrapped x copies)
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            T* ps = sm + s * rows * W + (R + ly) * W;
            const T v = q[s][R];
            ps[R + ix] = v;
            if (ix < R) ps[R + nx + ix] = v;
            if (ix >= nx - R) ps[ix - (nx - R)] = v;
        }
        // halo rows above and below the tile (wrapped in y)
        const long long zoff = (long long)z * plane;
        for (int h = t; h < 2 * R * nx; h += blockDim.x) {
            const int hr = h / nx, hx = h % nx;
            const int src = wrap_idx(hr < R ? y0 - R + hr : y0 + ty + (hr - R), ny);
            const int dst = hr < R ? hr : ty + hr;
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
                const T v = Xs[s][zoff + (long long)src * nx + hx];
                T* ps = sm + s * rows * W + dst * W;
                ps[R + hx] = v;
                if (hx < R) ps[R + nx + hx] = v;
                if (hx >= nx - R) ps[hx - (nx - R)] = v;
            }
        }
        __syncthreads();

        const long long gi = zoff + col;
        const T vloc = a.V[gi];
        T nl[SPB];
#pragma unroll
        for (int s = 0; s < SPB; ++s) nl[s] = T(0);
        if (a.row) {
            const int e0 = a.row[gi], e1 = a.row[gi + 1];
            for (int e = e0; e < e1; ++e) {
                const int at = a.ent_atom[e];
                const T* ev = a.ent_val + (long long)e * a.nch;
                for (int ch = 0; ch < a.nch; ++ch) {
                    const T tv = ev[ch];
#pragma unroll
                    for (int s = 0; s < SPB; ++s)
                        nl[s] += tv * a.coef[(long long)(at * a.nch + ch) * a.ldc + (valid[s] ? s0 + s : s0)];
                }
            }
        }
#pragma unroll
        for (int s = 0; s < SPB; ++s) {
            const T* pc = sm + s * rows * W + (R + ly) * W + R + ix;
            const T lap = stencil_point<T, ORDER, R>(pc, W, q[s], a);
            const T out = (vloc * q[s][R] + nl[s]) + lap;
            if (valid[s]) a.HX[(long long)(s0 + s) * a.ldhx + gi] = out;
        }
        __syncthreads();
        if (more) {
#pragma unroll
            for (int s = 0; s < SPB; ++s) {
#pragma unroll
                for (int d = 0; d < Q - 1; ++d) q[s][d] = q[s][d + 1];
                q[s][Q - 1] = nq[s];
            }
        }
    }
}

// Gather-contraction of the projectors. `chunks` blocks serve one (atom, group of
// SB states) as a thread-block cluster: block r sums the r-th contiguous part of the
// atom's sphere points, the partial sums meet in block 0 through distributed shared
// memory and are added in rank order. The split depends only on the cell (never on
// the number of states), so an apply gives the same bits for a state whatever batch
// it is in. Splitting an atom shortens each block's serial walk over its points
// (latency-bound for small cells) and keeps all atoms of one state group on the GPU
// together, so their overlapping spheres are gathered from L2.
// The coefficients are stored channel-major, coef[(atom * NCH + ch) * ldc + s], so
// that the scatter reads the states of one (atom, channel) as contiguous vectors.
__device__ __forceinline__ uint32_t smem_u32addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Asynchronous gather of one element into shared memory (no register holds it in flight).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32addr(smem)), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

constexpr int kProjThreads = 256;
// DEPTH > 0: the states at a point and its table values are gathered with cp.async into
// a DEPTH-stage ring of per-thread shared-memory slots (each thread reads back only its
// own slots, so no block barrier), the grid indices DEPTH points ahead in registers:
// DEPTH - 1 points' gathers stay in flight without holding registers. The points of a
// thread and the order of its sums are those of the register path (DEPTH = 0), so the
// result is the same to the bit.
template <typename T, int SB, int NCH, int DEPTH>
__global__ void __launch_bounds__(kProjThreads) k_project(const T* __restrict__ X, long long ldx, int ns,
                                                 const int* __restrict__ atom_off,
                                                 const int* __restrict__ pt_g,
                                                 const T* __restrict__ tab, long long npts,
                                                 const double* __restrict__ ch_scale,
                                                 T* __restrict__ coef, long long ldc, int chunks) {
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int atom = blockIdx.x / chunks;
    const int a0 = atom_off[atom], a1 = atom_off[atom + 1];
    const int len = (a1 - a0 + chunks - 1) / chunks;
    const int p0 = min(a1, a0 + rank * len), p1 = min(a1, p0 + len);
    const int s0 = blockIdx.y * SB;
    T acc[SB][NCH];
#pragma unroll
    for (int s = 0; s < SB; ++s)
#pragma unroll
        for (int c = 0; c < NCH; ++c) acc[s][c] = T(0);
    const T* Xs[SB];  // states past the end read the last valid state
#pragma unroll
    for (int s = 0; s < SB; ++s) Xs[s] = X + (long long)min(s0 + s, ns - 1) * ldx;

    if constexpr (DEPTH > 0) {
        extern __shared__ __align__(16) unsigned char proj_dsm[];
        T* ring = reinterpret_cast<T*>(proj_dsm);  // [DEPTH][SB + NCH][kProjThreads]
        const int tid = threadIdx.x;
        auto slot = [&](int d, int q) { return ring + ((size_t)d * (SB + NCH) + q) * kProjThreads + tid; };
        auto issue = [&](int d, int g, int pt) {
#pragma unroll
            for (int s = 0; s < SB; ++s) cp_async_elem(slot(d, s), Xs[s] + g);
#pragma unroll
            for (int c = 0; c < NCH; ++c) cp_async_elem(slot(d, SB + c), tab + (long long)c * npts + pt);
        };
        const int niter = (p1 - p0 + kProjThreads - 1) / kProjThreads;  // the same for the whole block
#pragma unroll
        for (int j = 0; j < DEPTH - 1; ++j) {
            const int pj = p0 + tid + j * kProjThreads;
            if (pj < p1) issue(j, pt_g[pj], pj);
            cp_async_commit();
        }
        int gq[DEPTH];
#pragma unroll
        for (int j = DEPTH - 1; j < 2 * DEPTH - 1; ++j) {
            const int pj = p0 + tid + j * kProjThreads;
            gq[j % DEPTH] = pj < p1 ? pt_g[pj] : 0;
        }
        for (int i0 = 0; i0 < niter; i0 += DEPTH) {
#pragma unroll
            for (int u = 0; u < DEPTH; ++u) {
                const int i = i0 + u;
                if (i < niter) {
                    const int sj = (u + DEPTH - 1) % DEPTH;  // slot of point i + DEPTH - 1
                    const int pj = p0 + tid + (i + DEPTH - 1) * kProjThreads;
                    if (pj < p1) issue(sj, gq[sj], pj);
                    const int pr = pj + DEPTH * kProjThreads;
                    gq[sj] = pr < p1 ? pt_g[pr] : 0;
                    cp_async_commit();
                    cp_async_wait<DEPTH - 1>();  // this thread's gathers of point i have landed
                    if (p0 + tid + i * kProjThreads < p1) {
                        T tv[NCH];
#pragma unroll
                        for (int c = 0; c < NCH; ++c) tv[c] = *slot(u, SB + c);
#pragma unroll
                        for (int s = 0; s < SB; ++s) {
                            const T v = *slot(u, s);
#pragma unroll
                            for (int c = 0; c < NCH; ++c) acc[s][c] += tv[c] * v;
                        }
                    }
                }
            }
        }
        cp_async_wait<0>();
    } else {
    // software pipeline: the grid index and table values of the next point are in
    // flight while the states are gathered at the current one, so each step waits
    // for one memory latency instead of two dependent ones
    int p = p0 + threadIdx.x;
    int g = 0;
    T tv[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) tv[c] = T(0);
    if (p < p1) {
        g = pt_g[p];
#pragma unroll
        for (int c = 0; c < NCH; ++c) tv[c] = tab[(long long)c * npts + p];
    }
#pragma unroll 2
    for (; p < p1; p += blockDim.x) {
        const int pn = p + blockDim.x;
        int gn = 0;
        T tn[NCH];
#pragma unroll
        for (int c = 0; c < NCH; ++c) tn[c] = T(0);
        if (pn < p1) {
            gn = pt_g[pn];
#pragma unroll
            for (int c = 0; c < NCH; ++c) tn[c] = tab[(long long)c * npts + pn];
        }
#pragma unroll
        for (int s = 0; s < SB; ++s) {
            const T v = Xs[s][g];
#pragma unroll
            for (int c = 0; c < NCH; ++c) acc[s][c] += tv[c] * v;
        }
        g = gn;
#pragma unroll
        for (int c = 0; c < NCH; ++c) tv[c] = tn[c];
    }
    }
    // block reduction: warp shuffles, then one value per warp through shared memory
    __shared__ T red[8][SB * NCH];
    __shared__ T part[SB * NCH];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < SB; ++s)
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            T v = acc[s][c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][c * SB + s] = v;
        }
    __syncthreads();
    const int nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < SB * NCH; i += blockDim.x) {
        T v = T(0);
        for (int w = 0; w < nw; ++w) v += red[w][i];
        part[i] = v;
    }
    cluster.sync();  // every part's sums are in its block's shared memory
    if (rank == 0) {
        for (int i = threadIdx.x; i < SB * NCH; i += blockDim.x) {
            T v = T(0);
            for (int r = 0; r < chunks; ++r) v += *cluster.map_shared_rank(&part[i], r);
            const int c = i / SB, s = i % SB;
            if (s0 + s < ns)
                coef[(long long)(atom * NCH + c) * ldc + s0 + s] = T(ch_scale[atom * NCH + c] * (double)v);
        }
    }
    cluster.sync();  // the other parts keep their shared memory until block 0 has read it
}

// States per projection block (or the forced value): the largest of 8 / 4 / 2 / 1
// that still gives one block per SM. 8 states measured fastest at 32-256 states on
// 64- and 216-atom cells (16 holds more registers than it saves table reads).
static int pick_project_sb(int blocks_per_group, int ns, int forced) {
    if (forced > 0) return forced;
    for (int sb : {8, 4, 2})
        if ((long long)blocks_per_group * ((ns + sb - 1) / sb) >= 148) return sb;
    return 1;
}

constexpr int kProjDepth = 3;  // cp.async stages of the projection's gather

template <typename T, int NCH>
static int launch_project_nch(const DevProjectors& pj, const T* tab, int ns, const T* X, long long ldx, T* coef,
                              long long ldc, int sb, int parts, cudaStream_t st, const double* scale) {
    // register budget: 16 states only with 4 channels, 8 with 8, 4 with 16
    constexpr int kMaxSb = NCH <= 4 ? 16 : (NCH == 8 ? 8 : 4);
    sb = std::min(sb, kMaxSb);
    const dim3 g(pj.na * parts, (ns + sb - 1) / sb);
    cudaError_t e;
#define QG_PROJECT(SBV)                                                                                        \
    do {                                                                                                       \
        const size_t smem = (size_t)kProjDepth * (SBV + NCH) * kProjThreads * sizeof(T);                       \
        auto kern = k_project<T, SBV, NCH, kProjDepth>;                                                        \
        if (allow_max_dynamic_smem(kern) != cudaSuccess) \
            return QG_ERR_CUDA;                                                                                \
        e = launch_clustered(kern, g, dim3(kProjThreads), parts, smem, st, X, ldx, ns, pj.atom_off, pj.pt_g,   \
                             tab, pj.npts, scale, coef, ldc, parts);                                           \
    } while (0)
    switch (sb) {
        case 16:
            if constexpr (kMaxSb >= 16) {
                QG_PROJECT(16);
                break;
            }
            [[fallthrough]];
        case 8:
            if constexpr (kMaxSb >= 8) {
                QG_PROJECT(8);
                break;
            }
            [[fallthrough]];
        case 4: QG_PROJECT(4); break;
        case 2: QG_PROJECT(2); break;
        default: QG_PROJECT(1); break;
    }
#undef QG_PROJECT
    QG_CUDA_TRY(e);
    return QG_OK;
}

// scale[atom * nch + ch] multiplies each sum (nullptr: E_k * dV, the operator's coefficients).
template <typename T>
static int launch_project(const DevProjectors& pj, int ns, const T* X, long long ldx, T* coef, long long ldc,
                          int forced_sb, int forced_parts, cudaStream_t st, const double* scale = nullptr) {
    const T* tab;
    if constexpr (sizeof(T) == 8) tab = reinterpret_cast<const T*>(pj.tab_d);
    else tab = reinterpret_cast<const T*>(pj.tab_f);
    if (!scale) scale = pj.ch_scale;
    const int parts = project_parts(pj, forced_parts);
    const int sb = pick_project_sb(pj.na * parts, ns, forced_sb);
    switch (pj.nch) {
        case 4: return launch_project_nch<T, 4>(pj, tab, ns, X, ldx, coef, ldc, sb, parts, st, scale);
        case 8: return launch_project_nch<T, 8>(pj, tab, ns, X, ldx, coef, ldc, sb, parts, st, scale);
        case 16: return launch_project_nch<T, 16>(pj, tab, ns, X, ldx, coef, ldc, sb, parts, st, scale);
        default: return QG_ERR_UNSUPPORTED;
    }
}

int project_inner_d(qg_hamiltonian h, int ns, const double* X, long long ldx, double* coef, long long ldc,
                    cudaStream_t st) {
    return launch_project<double>(h->pj, ns, X, ldx, coef, ldc, h->proj_sb, h->proj_parts, st, h->pj.ch_dv);
}

// 16-byte vector of T (the unit the scatter reads the coefficients in).
template <typename T> struct Vec16;
template <> struct Vec16<double> {
    using type = double2;
    static constexpr int n = 2;
    static __device__ __forceinline__ double at(const double2& v, int i) { return i == 0 ? v.x : v.y; }
};
template <> struct Vec16<float> {
    using type = float4;
    static constexpr int n = 4;
    static __device__ __forceinline__ float at(const float4& v, int i) {
        return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
    }
};

// Nonlocal scatter over all states, one thread per grid point. The point's first
// KMAX entries (their coefficient rows and NCH table values) stay in registers for
// all state groups; for each group of SG states every entry adds
// sum_ch val[ch] * coef[atom, ch][s0 .. s0+SG), read as 16-byte vectors (the lanes of
// a warp mostly share the entry's atom, so these are broadcast loads from L1).
// Entries past KMAX (points inside more than KMAX spheres) are read from memory in
// the same order, so the sum per point and state is the same as one loop over all.
template <typename T, int SG, int NCH, int KMAX>
__global__ void __launch_bounds__(256, SG <= 4 ? 3 : 2) k_scatter_all(T* __restrict__ HX, long long ldhx, int ns, long long N,
                                                     const int* __restrict__ row,
                                                     const int* __restrict__ ent_atom,
                                                     const T* __restrict__ ent_val,
                                                     const T* __restrict__ coef, long long ldc) {
    using V = typename Vec16<T>::type;
    constexpr int VN = Vec16<T>::n;
    static_assert(SG % VN == 0, "state group must be whole vectors");
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N) return;
    const int e0 = row[g], ne = row[g + 1] - e0;
    if (ne == 0) return;
    int cb[KMAX];  // first coefficient row of the entry's atom
    T v[KMAX][NCH];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        cb[k] = 0;
#pragma unroll
        for (int c = 0; c < NCH; ++c) v[k][c] = T(0);
        if (k < ne) {
            cb[k] = __ldg(&ent_atom[e0 + k]) * NCH;
#pragma unroll
            for (int c = 0; c < NCH; ++c) v[k][c] = __ldg(&ent_val[(long long)(e0 + k) * NCH + c]);
        }
    }
    for (int s0 = 0; s0 < ns; s0 += SG) {
        // the group's H psi values load first, so their latency overlaps the sums
        const int gn = min(SG, ns - s0);
        T h[SG];
#pragma unroll
        for (int s = 0; s < SG; ++s) h[s] = (s < gn) ? HX[(long long)(s0 + s) * ldhx + g] : T(0);
        T acc[SG];
#pragma unroll
        for (int s = 0; s < SG; ++s) acc[s] = T(0);
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
            if (k < ne) {
#pragma unroll
                for (int c = 0; c < NCH; ++c) {
                    const V* cp = reinterpret_cast<const V*>(coef + (long long)(cb[k] + c) * ldc + s0);
#pragma unroll
                    for (int j = 0; j < SG / VN; ++j) {
                        const V w = __ldg(cp + j);
#pragma unroll
                        for (int i = 0; i < VN; ++i) acc[j * VN + i] += v[k][c] * Vec16<T>::at(w, i);
                    }
                }
            }
        }
        for (int e = e0 + KMAX; e < e0 + ne; ++e) {
            const T* ce = coef + (long long)__ldg(&ent_atom[e]) * NCH * ldc;
#pragma unroll
            for (int c = 0; c < NCH; ++c) {
                const T vc = __ldg(&ent_val[(long long)e * NCH + c]);
                const V* cp = reinterpret_cast<const V*>(ce + (long long)c * ldc + s0);
#pragma unroll
                for (int j = 0; j < SG / VN; ++j) {
                    const V w = __ldg(cp + j);
#pragma unroll
                    for (int i = 0; i < VN; ++i) acc[j * VN + i] += vc * Vec16<T>::at(w, i);
                }
            }
        }
#pragma unroll
        for (int s = 0; s < SG; ++s)
            if (s < gn) HX[(long long)(s0 + s) * ldhx + g] = h[s] + acc[s];
    }
}

template <typename T, int NCH>
static int launch_scatter_all_nch(const DevProjectors& pj, T* HX, long long ldhx, int ns, long long N,
                                  const T* coef, long long ldc, int sg, cudaStream_t st) {
    constexpr int KMAX = NCH <= 4 ? 3 : (NCH == 8 ? 2 : 1);
    const T* ev;
    if constexpr (sizeof(T) == 8) ev = reinterpret_cast<const T*>(pj.ent_val_d);
    else ev = reinterpret_cast<const T*>(pj.ent_val_f);
    const unsigned grid = (unsigned)((N + 255) / 256);
    if (sg == 4)
        k_scatter_all<T, 4, NCH, KMAX><<<grid, 256, 0, st>>>(HX, ldhx, ns, N, pj.row, pj.ent_atom, ev, coef, ldc);
    else
        k_scatter_all<T, 8, NCH, KMAX><<<grid, 256, 0, st>>>(HX, ldhx, ns, N, pj.row, pj.ent_atom, ev, coef, ldc);
    return QG_OK;
}

template <typename T>
static int launch_scatter_all(const DevProjectors& pj, T* HX, long long ldhx, int ns, long long N, const T* coef,
                              long long ldc, int forced_sg, cudaStream_t st) {
    const int sg = forced_sg == 4 ? 4 : 8;
    switch (pj.nch) {
        case 4: return launch_scatter_all_nch<T, 4>(pj, HX, ldhx, ns, N, coef, ldc, sg, st);
        case 8: return launch_scatter_all_nch<T, 8>(pj, HX, ldhx, ns, N, coef, ldc, sg, st);
        case 16: return launch_scatter_all_nch<T, 16>(pj, HX, ldhx, ns, N, coef, ldc, sg, st);
        default: return QG_ERR_UNSUPPORTED;
    }
}

template <typename T, int ORDER>
static int launch_stencil(const HamArgs<T>& a, int nz, cudaStream_t st) {
    constexpr int R = ORDER == 2 ? 1 : (ORDER == 8 ? 4 : 3);
    constexpr int SPB = 1;
    const int tiles = a.ny / a.ty;
    const int sgroups = (a.ns + SPB - 1) / SPB;
    // enough blocks for every SM: split z into slabs when the (tile, state) grid is small
    long long base = (long long)tiles * sgroups;
    int nslab = 1;
    const long long target = 4LL * 148;
    if (base < target) nslab = (int)std::min<long long>((target + base - 1) / base, std::max(1, nz / (2 * R)));
    HamArgs<T> b = a;
    b.zslab = (nz + nslab - 1) / nslab;
    nslab = (nz + b.zslab - 1) / b.zslab;
    const size_t smem = (size_t)SPB * (a.ty + 2 * R) * (a.nx + 2 * R) * sizeof(T);
    auto kern = k_hamiltonian<T, ORDER, SPB>;
    if (smem > 48 * 1024) {
        if (allow_max_dynamic_smem(kern) != cudaSuccess)
            return QG_ERR_UNSUPPORTED;
    }
    dim3 grid(tiles, sgroups, nslab);
    kern<<<grid, a.nx * a.ty, smem, st>>>(b);
    return QG_OK;
}

size_t coef_scratch_elems(qg_hamiltonian h, int ns) {
    const DevProjectors& pj = h->pj;
    if (pj.na <= 0 || pj.nch <= 0) return 0;
    return (size_t)coef_ld(ns) * pj.na * pj.nch;
}

size_t coef_scratch_elems_z(qg_hamiltonian h, int nk, int nsk) {
    const DevProjectors& pj = h->pj;
    if (pj.na <= 0 || pj.nch <= 0) return 0;
    return (size_t)2 * nk * coef_ld(nsk) * pj.na * pj.nch;
}

// Stencil kernel for a real-state apply: the forced variant when it accepts the shape,
// else the two-row ring kernel -- FP64 with V in the ring (4), FP32 with V from global
// memory (5) -- measured on the 80^3 cell, 256 states (whole apply, order 2/4/6/8):
// FP64 4: 1.46/1.52/1.52/1.55 ms, 5: 1.58/1.59/1.59/1.59, one-plane (2): 1.52/1.75/1.77/1.77;
// FP32 5: 0.87/1.03/1.03/1.10, 4: 1.00/1.06/1.04/1.11, 2: 0.91/1.11/1.10/1.12;
// then the other ring kernels, else (1) the register-window kernel, which takes any
// shape. All ring kernels give the same bits.
template <typename T>
static int ring_stencil_variant(qg_hamiltonian h, const HamArgs<T>& a) {
    const int v = h->stencil_variant;
    if (v == 1) return 1;
    const bool pair_ok = stencil_pair_ok<T>(a, h->order);
    const bool tma_ok = stencil_tma_ok<T>(a, h->order);
    const bool rows_ok = stencil_rows_ok<T>(a, h->order, true);
    const bool rowsg_ok = stencil_rows_ok<T>(a, h->order, false);
    if (v == 3 && pair_ok) return 3;
    if (v == 2 && tma_ok) return 2;
    if (v == 4 && rows_ok) return 4;
    if (v == 5 && rowsg_ok) return 5;
    if (sizeof(T) == 4 && rowsg_ok) return 5;
    if (rows_ok) return 4;
    if (rowsg_ok) return 5;
    if (tma_ok) return 2;
    if (pair_ok) return 3;
    return 1;
}

template <typename T>
int apply_hamiltonian(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx,
                      T* coef, cudaStream_t st, PhaseTimer* pt) {
    const DevProjectors& pj = h->pj;
    HamArgs<T> a{};
    a.X = X; a.ldx = ldx; a.HX = HX; a.ldhx = ldhx; a.ns = ns;
    if constexpr (sizeof(T) == 8) a.V = reinterpret_cast<const T*>(h->V_d);
    else a.V = reinterpret_cast<const T*>(h->V_f);
    a.nx = h->nx; a.ny = h->ny; a.nz = h->nz; a.ty = h->ty;
    // coefficients of -1/2 Lap exactly as the reference forms them
    const double coefk = -0.5;
    const double ih[3] = {h->hx, h->hy, h->hz};
    T* cs[3] = {a.cx, a.cy, a.cz};
    switch (h->order) {
        case 2:
            a.c0 = T(-coefk * (2.0 / (ih[0] * ih[0]) + 2.0 / (ih[1] * ih[1]) + 2.0 / (ih[2] * ih[2])));
            for (int d = 0; d < 3; ++d) cs[d][0] = T(coefk / (ih[d] * ih[d]));
            break;
        case 4:
            for (int d = 0; d < 3; ++d) {
                const double s = (24.0 * ih[d]) * (24.0 * ih[d]);
                cs[d][2] = T(coefk / s);
                cs[d][1] = T(-54.0 * coefk / s);
                cs[d][0] = T(783.0 * coefk / s);
            }
            break;
        case 6:
            a.c0 = T(-245.0 * coefk * (1.0 / (90.0 * ih[0] * ih[0]) + 1.0 / (90.0 * ih[1] * ih[1]) + 1.0 / (90.0 * ih[2] * ih[2])));
            for (int d = 0; d < 3; ++d) {
                const double s = 90.0 * ih[d] * ih[d];
                cs[d][2] = T(coefk / s);
                cs[d][1] = T(-13.5 * coefk / s);
                cs[d][0] = T(135.0 * coefk / s);
            }
            break;
        case 8:
            a.c0 = T(-14350.0 / 5040.0 * coefk * (1.0 / (ih[0] * ih[0]) + 1.0 / (ih[1] * ih[1]) + 1.0 / (ih[2] * ih[2])));
            for (int d = 0; d < 3; ++d) {
                const double s = 5040.0 * ih[d] * ih[d];
                cs[d][3] = T(-9.0 * coefk / s);
                cs[d][2] = T(128.0 * coefk / s);
                cs[d][1] = T(-1008.0 * coefk / s);
                cs[d][0] = T(8064.0 * coefk / s);
            }
            break;
        default: return QG_ERR_INVALID;
    }
    a.err = h->ctx->dev_status;
    a.stall = h->test_stall;
    const bool nonlocal = pj.na > 0 && pj.nch > 0;
    const long long N = h->N();
    const int variant = ring_stencil_variant<T>(h, a);
    if (variant != 1) {
        auto stencil = [&]() {
            if (variant == 3) return launch_stencil_pair<T>(a, h->order, st);
            if (variant == 4) return launch_stencil_rows<T>(a, h->order, st, true);
            if (variant == 5) return launch_stencil_rows<T>(a, h->order, st, false);
            return launch_stencil_tma<T>(a, h->order, st);
        };
        if (!nonlocal) {
            if (pt) pt->mark(1, st);
            QG_TRY(stencil());
            QG_CUDA_TRY(cudaGetLastError());
            if (pt) pt->mark(-1, st);
            return QG_OK;
        }
        // projection of all states, persistent stencil + V, then the nonlocal scatter
        if (pt) pt->mark(0, st);
        QG_TRY(launch_project<T>(pj, ns, X, ldx, coef, coef_ld(ns), h->proj_sb, h->proj_parts, st));
        if (pt) pt->mark(1, st);
        QG_TRY(stencil());
        if (pt) pt->mark(2, st);
        QG_TRY(launch_scatter_all<T>(pj, HX, ldhx, ns, N, coef, coef_ld(ns), h->scatter_sg, st));
        if (pt) pt->mark(-1, st);
        QG_CUDA_TRY(cudaGetLastError());
        return QG_OK;
    }
    // register-window kernel with the nonlocal scatter fused per point
    if (pt) pt->mark(0, st);
    if (nonlocal) {
        QG_TRY(launch_project<T>(pj, ns, X, ldx, coef, coef_ld(ns), h->proj_sb, h->proj_parts, st));
        a.row = pj.row;
        a.ent_atom = pj.ent_atom;
        if constexpr (sizeof(T) == 8) a.ent_val = reinterpret_cast<const T*>(pj.ent_val_d);
        else a.ent_val = reinterpret_cast<const T*>(pj.ent_val_f);
        a.nch = pj.nch;
        a.ldc = coef_ld(ns);
        a.coef = coef;
    }
    if (pt) pt->mark(1, st);
    int rc;
    switch (h->order) {
        case 2: rc = launch_stencil<T, 2>(a, h->nz, st); break;
        case 4: rc = launch_stencil<T, 4>(a, h->nz, st); break;
        case 6: rc = launch_stencil<T, 6>(a, h->nz, st); break;
        default: rc = launch_stencil<T, 8>(a, h->nz, st); break;
    }
    if (rc != QG_OK) return rc;
    if (pt) pt->mark(-1, st);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

template int apply_hamiltonian<double>(qg_hamiltonian, int, const double*, long long, double*,
                                       long long, double*, cudaStream_t, PhaseTimer*);
template int apply_hamiltonian<float>(qg_hamiltonian, int, const float*, long long, float*,
                                      long long, float*, cudaStream_t, PhaseTimer*);

}  // namespace qg

// --------------------------------------------------------------------------
// Host-side table building (once per geometry).

namespace {

int wrap_host(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

template <typename T>
int upload(T** dst, const std::vector<T>& src) {
    *dst = nullptr;
    if (src.empty()) return QG_OK;
    QG_CUDA_TRY(cudaMalloc(dst, src.size() * sizeof(T)));
    QG_CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return QG_OK;
}

void free_projectors(DevProjectors& pj) {
    cudaFree(pj.atom_off); cudaFree(pj.pt_g); cudaFree(pj.tab_d); cudaFree(pj.tab_f);
    cudaFree(pj.ch_scale); cudaFree(pj.ch_dv); cudaFree(pj.ch_E); cudaFree(pj.row); cudaFree(pj.ent_atom); cudaFree(pj.ent_val_d);
    cudaFree(pj.ent_val_f); cudaFree(pj.pt_u); cudaFree(pj.ent_pt); cudaFree(pj.ztab); cudaFree(pj.zent);
    cudaFree(pj.ztab_f); cudaFree(pj.zent_f);
    pj = DevProjectors();
}

// Compacts the reference's per-atom cube tables into sphere point lists and the
// per-grid-point entry list (see DevProjectors). A cube point is kept when any
// channel value is nonzero; points outside every cutoff hold exact zeros in the
// reference tables and add nothing.
int build_projectors(qg_hamiltonian h, const qg_hamiltonian_desc* d) {
    const int na = d->n_atoms, np = d->n_proj;
    if (na <= 0 || np <= 0) return QG_OK;
    int nch_real = 0;
    for (int k = 0; k < np; ++k) {
        if (d->proj_l[k] < 0 || d->proj_l[k] > 3) return QG_ERR_INVALID;
        nch_real += 2 * d->proj_l[k] + 1;
    }
    int nch = nch_real <= 4 ? 4 : (nch_real <= 8 ? 8 : (nch_real <= 16 ? 16 : -1));
    if (nch < 0) return QG_ERR_UNSUPPORTED;
    const double Y00 = 1.0 / sqrt(4.0 * M_PI);
    const double dV = h->hx * h->hy * h->hz;
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const long long N = h->N();

    std::vector<int> atom_off(na + 1, 0);
    std::vector<int> pt_g, pt_u;
    std::vector<std::vector<double>> tabs(nch);
    std::vector<double> ch_scale((size_t)na * nch, 0.0), ch_dv((size_t)na * nch, 0.0), ch_E((size_t)na * nch, 0.0);
    std::vector<int> ch_k(nch, -1), ch_m(nch, 0);
    {
        int c = 0;
        for (int k = 0; k < np; ++k)
            for (int m = 0; m < 2 * d->proj_l[k] + 1; ++m) { ch_k[c] = k; ch_m[c] = m; ++c; }
    }
    for (int a = 0; a < na; ++a) {
        int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
        for (int k = 0; k < np; ++k) {
            const int* c = d->cube + 6 * ((size_t)a * np + k);
            for (int i = 0; i < 3; ++i) {
                if (c[3 + i] <= 0) return QG_ERR_INVALID;
                lo[i] = std::min(lo[i], c[i]);
                hi[i] = std::max(hi[i], c[i] + c[3 + i]);
            }
        }
        for (int ch = 0; ch < nch; ++ch) {
            ch_scale[(size_t)a * nch + ch] = ch_k[ch] >= 0 ? d->proj_E[ch_k[ch]] * dV : 0.0;
            ch_dv[(size_t)a * nch + ch] = ch_k[ch] >= 0 ? dV : 0.0;
            ch_E[(size_t)a * nch + ch] = ch_k[ch] >= 0 ? d->proj_E[ch_k[ch]] : 0.0;
        }
        std::vector<double> vals(nch);
        for (int z = lo[2]; z < hi[2]; ++z)
            for (int y = lo[1]; y < hi[1]; ++y)
                for (int x = lo[0]; x < hi[0]; ++x) {
                    bool any = false;
                    for (int ch = 0; ch < nch; ++ch) {
                        vals[ch] = 0.0;
                        const int k = ch_k[ch];
                        if (k < 0) continue;
                        const int* c = d->cube + 6 * ((size_t)a * np + k);
                        const int qx = x - c[0], qy = y - c[1], qz = z - c[2];
                        if (qx < 0 || qy < 0 || qz < 0 || qx >= c[3] || qy >= c[4] || qz >= c[5]) continue;
                        const size_t q = qx + (size_t)c[3] * (qy + (size_t)c[4] * qz);
                        const double w = d->w_data[d->w_off[(size_t)a * np + k] + q];
                        const int l = d->proj_l[k];
                        if (l == 0) {
                            vals[ch] = w * Y00;
                        } else {
                            const int lm = l * l + ch_m[ch];
                            if (lm >= d->n_lm) return QG_ERR_INVALID;
                            vals[ch] = w * d->ylm_data[d->ylm_off[(size_t)a * d->n_lm + lm] + q];
                        }
                        if (vals[ch] != 0.0) any = true;
                    }
                    if (!any) continue;
                    const long long g = wrap_host(x, nx) + (long long)nx * (wrap_host(y, ny) + (long long)ny * wrap_host(z, nz));
                    pt_g.push_back((int)g);
                    pt_u.push_back(x); pt_u.push_back(y); pt_u.push_back(z);
                    for (int ch = 0; ch < nch; ++ch) tabs[ch].push_back(vals[ch]);
                }
        atom_off[a + 1] = (int)pt_g.size();
    }
    const long long npts = (long long)pt_g.size();
    std::vector<double> tab_d((size_t)nch * npts);
    for (int ch = 0; ch < nch; ++ch) std::copy(tabs[ch].begin(), tabs[ch].end(), tab_d.begin() + (size_t)ch * npts);
    std::vector<float> tab_f(tab_d.begin(), tab_d.end());

    // scatter side: per grid point, the (atom, values) entries covering it, atom-ordered
    std::vector<int> row(N + 1, 0);
    for (long long p = 0; p < npts; ++p) row[pt_g[p] + 1]++;
    for (long long g = 0; g < N; ++g) row[g + 1] += row[g];
    std::vector<int> fill(row.begin(), row.end() - 1);
    std::vector<int> ent_atom(npts), ent_pt(npts);
    std::vector<double> ent_val((size_t)npts * nch);
    for (int a = 0; a < na; ++a)
        for (int p = atom_off[a]; p < atom_off[a + 1]; ++p) {
            const int e = fill[pt_g[p]]++;
            ent_atom[e] = a;
            ent_pt[e] = p;
            for (int ch = 0; ch < nch; ++ch) ent_val[(size_t)e * nch + ch] = tab_d[(size_t)ch * npts + p];
        }
    std::vector<float> ent_val_f(ent_val.begin(), ent_val.end());

    DevProjectors& pj = h->pj;
    pj.na = na; pj.nch = nch; pj.npts = npts; pj.nent = npts;
    pj.max_atom_pts = 0;
    for (int a = 0; a < na; ++a) pj.max_atom_pts = std::max<long long>(pj.max_atom_pts, atom_off[a + 1] - atom_off[a]);
    QG_TRY(upload(&pj.atom_off, atom_off));
    QG_TRY(upload(&pj.pt_g, pt_g));
    QG_TRY(upload(&pj.tab_d, tab_d));
    QG_TRY(upload(&pj.tab_f, tab_f));
    QG_TRY(upload(&pj.ch_scale, ch_scale));
    QG_TRY(upload(&pj.ch_dv, ch_dv));
    QG_TRY(upload(&pj.ch_E, ch_E));
    QG_TRY(upload(&pj.row, row));
    QG_TRY(upload(&pj.ent_atom, ent_atom));
    QG_TRY(upload(&pj.ent_val_d, ent_val));
    QG_TRY(upload(&pj.ent_val_f, ent_val_f));
    QG_TRY(upload(&pj.pt_u, pt_u));
    QG_TRY(upload(&pj.ent_pt, ent_pt));
    return QG_OK;
}

void destroy_ham(qg_hamiltonian h) {
    if (!h) return;
    delete h->precond;
    cudaFree(h->V_d);
    cudaFree(h->V_f);
    free_projectors(h->pj);
    h->coef.release();
    h->kco.release();
    h->scf_work.release();
    if (h->io_in) cudaStreamDestroy(h->io_in);
    if (h->io_out) cudaStreamDestroy(h->io_out);
    h->xio.release();
    h->hxio.release();
    delete h;
}

}  // namespace

extern "C" {

int qg_hamiltonian_create(qg_context ctx, const qg_hamiltonian_desc* d, qg_hamiltonian* out) {
    if (!ctx || !d || !out) return QG_ERR_INVALID;
    *out = nullptr;
    if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || !(d->hx > 0) || !(d->hy > 0) || !(d->hz > 0) || !d->V)
        return QG_ERR_INVALID;
    const int R = qg::stencil_radius(d->fd_order);
    if (R < 0) return QG_ERR_INVALID;
    if (d->nx < 2 * R || d->ny < 2 * R || d->nz < 2 * R) return QG_ERR_UNSUPPORTED;
    if ((long long)d->nx * d->ny * d->nz >= (1LL << 31)) return QG_ERR_UNSUPPORTED;
    const int ty = qg::pick_tile_rows(d->nx, d->ny);
    if (ty <= 0) return QG_ERR_UNSUPPORTED;
    if (d->n_atoms > 0 && d->n_proj > 0 &&
        (!d->proj_l || !d->proj_E || !d->cube || !d->w_data || !d->w_off || !d->ylm_off))
        return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    qg_hamiltonian h = new qg_hamiltonian_s();
    h->ctx = ctx;
    h->nx = d->nx; h->ny = d->ny; h->nz = d->nz;
    h->hx = d->hx; h->hy = d->hy; h->hz = d->hz;
    h->order = d->fd_order;
    h->gx = d->gx; h->gy = d->gy; h->gz = d->gz;
    h->ty = ty;
    const long long N = h->N();
    std::vector<double> V(d->V, d->V + N);
    std::vector<float> Vf(V.begin(), V.end());
    int rc = upload(&h->V_d, V);
    if (rc == QG_OK) rc = upload(&h->V_f, Vf);
    if (rc == QG_OK) rc = build_projectors(h, d);
    if (rc != QG_OK) {
        destroy_ham(h);
        return rc;
    }
    ctx->live_hamiltonians++;
    *out = h;
    return QG_OK;
}

int qg_hamiltonian_destroy(qg_hamiltonian h) {
    if (!h) return QG_ERR_INVALID;
    cudaSetDevice(h->ctx->device);
    cudaStreamSynchronize(h->ctx->stream);
    h->ctx->live_hamiltonians--;
    destroy_ham(h);
    return QG_OK;
}

int qg_hamiltonian_set_kvector(qg_hamiltonian h, double gx, double gy, double gz) {
    if (!h) return QG_ERR_INVALID;
    h->gx = gx; h->gy = gy; h->gz = gz;
    return QG_OK;
}

}  // extern "C"

template <typename T>
static int apply_device(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx) {
    if (!h || ns < 0 || (ns > 0 && (!X || !HX))) return QG_ERR_INVALID;
    if (ns == 0) return QG_OK;
    const long long N = h->N();
    if (ldx < N || ldhx < N) return QG_ERR_INVALID;
    if (h->gx != 0.0 || h->gy != 0.0 || h->gz != 0.0) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    T* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems(h, ns) * sizeof(T)));
        coef = h->coef.as<T>();
    }
    return qg::apply_hamiltonian<T>(h, ns, X, ldx, HX, ldhx, coef, h->ctx->stream);
}

namespace qg {

int host_pipelined_apply(qg_hamiltonian h, int ns, long long row, const double* X, double* HX,
                         const std::function<int(int, const double*, double*)>& apply) {
    const size_t bytes = (size_t)ns * row * sizeof(double);
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    QG_TRY(h->xio.reserve(bytes));
    QG_TRY(h->hxio.reserve(bytes));
    if (!h->io_in) QG_CUDA_TRY(cudaStreamCreateWithFlags(&h->io_in, cudaStreamNonBlocking));
    if (!h->io_out) QG_CUDA_TRY(cudaStreamCreateWithFlags(&h->io_out, cudaStreamNonBlocking));
    cudaStream_t st = h->ctx->stream;
    // chunks of states: the copy-in of later chunks (io_in) and the copy-out of
    // earlier ones (io_out) run on both directions of the host link while the
    // apply of the current chunk runs on the context stream
    const int chunk = std::max(1, (ns + kHostChunks - 1) / kHostChunks);
    const int nchunk = (ns + chunk - 1) / chunk;
    std::vector<cudaEvent_t> ev(2 * nchunk + 1, nullptr);
    int rc = QG_OK;
    for (auto& e : ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) rc = QG_ERR_CUDA;
    // the copies start after the work already queued on the context stream
    if (rc == QG_OK && (cudaEventRecord(ev[2 * nchunk], st) != cudaSuccess ||
                        cudaStreamWaitEvent(h->io_in, ev[2 * nchunk], 0) != cudaSuccess ||
                        cudaStreamWaitEvent(h->io_out, ev[2 * nchunk], 0) != cudaSuccess))
        rc = QG_ERR_CUDA;
    double* xs = h->xio.as<double>();
    double* hs = h->hxio.as<double>();
    for (int c = 0; c < nchunk && rc == QG_OK; ++c) {
        const size_t off = (size_t)c * chunk * row;
        const size_t cb = (size_t)std::min(chunk, ns - c * chunk) * row * sizeof(double);
        if (cudaMemcpyAsync(xs + off, X + off, cb, cudaMemcpyHostToDevice, h->io_in) != cudaSuccess ||
            cudaEventRecord(ev[2 * c], h->io_in) != cudaSuccess)
            rc = QG_ERR_CUDA;
    }
    for (int c = 0; c < nchunk && rc == QG_OK; ++c) {
        const int nc = std::min(chunk, ns - c * chunk);
        const size_t off = (size_t)c * chunk * row;
        if (cudaStreamWaitEvent(st, ev[2 * c], 0) != cudaSuccess) {
            rc = QG_ERR_CUDA;
            break;
        }
        rc = apply(nc, xs + off, hs + off);
        if (rc != QG_OK) break;
        if (cudaEventRecord(ev[2 * c + 1], st) != cudaSuccess ||
            cudaStreamWaitEvent(h->io_out, ev[2 * c + 1], 0) != cudaSuccess ||
            cudaMemcpyAsync(HX + off, hs + off, (size_t)nc * row * sizeof(double), cudaMemcpyDeviceToHost,
                            h->io_out) != cudaSuccess)
            rc = QG_ERR_CUDA;
    }
    const cudaError_t e0 = cudaStreamSynchronize(h->io_in);
    const cudaError_t e1 = cudaStreamSynchronize(h->io_out);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    for (auto e : ev)
        if (e) cudaEventDestroy(e);
    if (rc != QG_OK) return rc;
    QG_CUDA_TRY(e0);
    QG_CUDA_TRY(e1);
    QG_CUDA_TRY(e2);
    return QG_OK;
}

}  // namespace qg

extern "C" {

int qg_hamiltonian_apply_d(qg_hamiltonian h, int ns, const double* X, long long ldx, double* HX,
                           long long ldhx) {
    return apply_device<double>(h, ns, X, ldx, HX, ldhx);
}

int qg_hamiltonian_apply_f(qg_hamiltonian h, int ns, const float* X, long long ldx, float* HX,
                           long long ldhx) {
    return apply_device<float>(h, ns, X, ldx, HX, ldhx);
}

int qg_hamiltonian_apply_timed_d(qg_hamiltonian h, int ns, const double* X, long long ldx,
                                 double* HX, long long ldhx, float* ms_phases) {
    if (!h || ns <= 0 || !X || !HX || !ms_phases) return QG_ERR_INVALID;
    const long long N = h->N();
    if (ldx < N || ldhx < N) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    double* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems(h, ns) * sizeof(double)));
        coef = h->coef.as<double>();
    }
    qg::PhaseTimer pt;
    const int rc = qg::apply_hamiltonian<double>(h, ns, X, ldx, HX, ldhx, coef, h->ctx->stream, &pt);
    if (rc != QG_OK) return rc;
    pt.totals(ms_phases);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int qg_hamiltonian_set_stencil_kernel(qg_hamiltonian h, int variant) {
    if (!h || variant < 0 || variant > 5) return QG_ERR_INVALID;
    h->stencil_variant = variant;
    return QG_OK;
}

int qg_hamiltonian_test_stall(qg_hamiltonian h, int on) {
    if (!h || (on != 0 && on != 1)) return QG_ERR_INVALID;
    h->test_stall = on;
    return QG_OK;
}

int qg_hamiltonian_set_nonlocal_blocking(qg_hamiltonian h, int project_states, int scatter_states,
                                         int project_parts) {
    if (!h) return QG_ERR_INVALID;
    const bool sb_ok = project_states == 0 || project_states == 1 || project_states == 2 || project_states == 4 ||
                       project_states == 8 || project_states == 16;
    const bool sg_ok = scatter_states == 0 || scatter_states == 4 || scatter_states == 8;
    const bool pp_ok = project_parts >= 0 && project_parts <= 8;
    if (!sb_ok || !sg_ok || !pp_ok) return QG_ERR_INVALID;
    h->proj_sb = project_states;
    h->scatter_sg = scatter_states;
    h->proj_parts = project_parts;
    return QG_OK;
}

int qg_hamiltonian_launches_per_apply(qg_hamiltonian h, int ns) {
    if (!h || ns < 0) return QG_ERR_INVALID;
    if (ns == 0) return 0;
    const bool nonlocal = h->pj.na > 0 && h->pj.nch > 0;
    qg::HamArgs<double> a{};
    a.X = reinterpret_cast<const double*>(16); a.HX = reinterpret_cast<double*>(16); a.V = h->V_d;
    a.ldx = a.ldhx = h->N(); a.nx = h->nx; a.ny = h->ny; a.nz = h->nz; a.err = h->ctx->dev_status;
    if (qg::ring_stencil_variant<double>(h, a) != 1) {
        if (!nonlocal) return 1;
        return 3;  // projection, stencil + V, nonlocal scatter
    }
    return (nonlocal ? 1 : 0) + 1;
}

int qg_hamiltonian_apply_host_d(qg_hamiltonian h, int ns, const double* X, double* HX) {
    if (!h || ns < 0 || (ns > 0 && (!X || !HX))) return QG_ERR_INVALID;
    if (ns == 0) return QG_OK;
    const long long N = h->N();
    return qg::host_pipelined_apply(h, ns, N, X, HX, [&](int nc, const double* xd, double* hd) {
        return apply_device<double>(h, nc, xd, N, hd, N);
    });
}

}  // extern "C"
