// Complex k-point Hamiltonian on the device (mHamiltonianMatrix_ddm of
// QUMASUN_KPOINT, qumasun_kpoint.matrix.h:25-50):
//   H_k u = V u + sum_atoms sum_k E_k sum_m conj(P_km) dV (P_km . u) - 1/2 (Lap + 2i g.grad - g^2) u,
//   P_km(r) = w_k(r) Y_lm(r) exp(i g.r) at the unwrapped image position of each cube point
//   (mCreateProjectorRadialOnBlock, PseudoPotOperator_kpoint_v2.h:287-420; ProjectionPP :2581-2700).
// States are split complex, one state = {re[N], im[N]} (lobpcg_z_multi_mpi.h:1005-1012).
// Three launches for a block of states, as on the real path:
//   k_project_z     c[k][a,ch][s] = E dV sum_p P(p) u_s(g(p))       (no conjugate, mInnerNonlocalPsi_v2)
//   k_stencil_tma   V u - 1/2 (Lap + 2i g.grad - g^2) u, both parts of a plane staged together
//                   (stencil_tma.cu, NC = 2); any other shape runs k_kpoint_plain
//   k_scatter_all_z Hu[s][g] += sum_entries conj(P) c                 (the scatter of ProjectionPP)
// The Bloch-phase tables are rebuilt on the device by k_bloch_tables whenever
// the k-vector differs from the one they were built for.
#include <algorithm>
#include <cmath>

#include <cooperative_groups.h>

#include "qg_internal.h"
#include "stencil_common.cuh"

namespace cg = cooperative_groups;

namespace qg {
namespace {

// ztab / zent for the k-vector g (see DevProjectors). theta = (ax ux + ay uy) + az uz,
// a* = g* h*, as the reference sums kxx + kyy + kzz.
// Computed in FP64 and stored as TO (FP64, or FP32 for complex64 states).
template <typename TO>
__global__ void k_bloch_tables(const double* __restrict__ tab, const int* __restrict__ pt_u, long long npts,
                               const int* __restrict__ ent_pt, long long nent, int nch, double ax, double ay,
                               double az, TO* __restrict__ ztab, TO* __restrict__ zent) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npts + nent; i += stride) {
        const long long p = i < npts ? i : ent_pt[i - npts];
        const double th = __dadd_rn(__dadd_rn(__dmul_rn(ax, (double)pt_u[3 * p]), __dmul_rn(ay, (double)pt_u[3 * p + 1])),
                                    __dmul_rn(az, (double)pt_u[3 * p + 2]));
        double sn, cs;
        sincos(th, &sn, &cs);
        if (i < npts) {
            for (int c = 0; c < nch; ++c) {
                const double v = tab[(long long)c * npts + p];
                ztab[(long long)c * npts + p] = TO(v * cs);
                ztab[(long long)(nch + c) * npts + p] = TO(v * sn);
            }
        } else {
            const long long e = i - npts;
            for (int c = 0; c < nch; ++c) {
                const double v = tab[(long long)c * npts + p];
                zent[(e * nch + c) * 2] = TO(v * cs);
                zent[(e * nch + c) * 2 + 1] = TO(v * sn);
            }
        }
    }
}

// Complex gather-contraction: one block per (atom, k-point, group of SB states).
// c = sum_p (tr + i ti)(ur + i ui), scaled by E dV per channel; the states of k-point k
// start at X + k*ldk, the Bloch tables of k at ztab + k*zstride. The coefficients are
// stored channel-major per k-point, {re, im} pairs at
// coef[((k * na * NCH + atom * NCH + ch) * ldc + s) * 2], so the scatter reads the
// states of one (k, atom, channel) as contiguous 16-byte pairs.
// As on the real path, `parts` blocks (a thread-block cluster) split each atom's
// points and add their partial sums in rank order through distributed shared memory.
template <typename T, int SB, int NCH>
__global__ void __launch_bounds__(256) k_project_z(const T* __restrict__ X, long long ldx, long long ldk,
                                                   long long xim, int nsk, int groups,
                                                   const int* __restrict__ atom_off, const int* __restrict__ pt_g,
                                                   const T* __restrict__ ztab, long long zstride, long long npts,
                                                   const double* __restrict__ ch_scale, T* __restrict__ coef,
                                                   int ncoef, long long ldc, int parts) {
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int atom = blockIdx.x / parts;
    const int k = blockIdx.y / groups;
    const int s0 = (blockIdx.y - k * groups) * SB;
    const int a0 = atom_off[atom], a1 = atom_off[atom + 1];
    const int len = (a1 - a0 + parts - 1) / parts;
    const int p0 = min(a1, a0 + rank * len), p1 = min(a1, p0 + len);
    const T* tab = ztab + (long long)k * zstride;
    T ar[SB][NCH], ai[SB][NCH];
#pragma unroll
    for (int s = 0; s < SB; ++s)
#pragma unroll
        for (int c = 0; c < NCH; ++c) ar[s][c] = ai[s][c] = T(0);
    const T* Xs[SB];
#pragma unroll
    for (int s = 0; s < SB; ++s) Xs[s] = X + (long long)k * ldk + (long long)min(s0 + s, nsk - 1) * ldx;

    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        const int g = pt_g[p];
        T tr[NCH], ti[NCH];
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            tr[c] = tab[(long long)c * npts + p];
            ti[c] = tab[(long long)(NCH + c) * npts + p];
        }
#pragma unroll
        for (int s = 0; s < SB; ++s) {
            const T ur = Xs[s][g], ui = Xs[s][xim + g];
#pragma unroll
            for (int c = 0; c < NCH; ++c) {
                ar[s][c] += tr[c] * ur - ti[c] * ui;
                ai[s][c] += ti[c] * ur + tr[c] * ui;
            }
        }
    }
    __shared__ T red[8][2 * SB * NCH];
    __shared__ T part[2 * SB * NCH];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < SB; ++s)
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            T vr = ar[s][c], vi = ai[s][c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                vr += __shfl_xor_sync(0xffffffffu, vr, o);
                vi += __shfl_xor_sync(0xffffffffu, vi, o);
            }
            if (lane == 0) {
                red[warp][2 * (s * NCH + c)] = vr;
                red[warp][2 * (s * NCH + c) + 1] = vi;
            }
        }
    __syncthreads();
    const int nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < 2 * SB * NCH; i += blockDim.x) {
        T v = T(0);
        for (int w = 0; w < nw; ++w) v += red[w][i];
        part[i] = v;
    }
    cluster.sync();  // every part's sums are in its block's shared memory
    if (rank == 0) {
        for (int i = threadIdx.x; i < 2 * SB * NCH; i += blockDim.x) {
            T v = T(0);
            for (int r = 0; r < parts; ++r) v += *cluster.map_shared_rank(&part[i], r);
            const int sc = i >> 1, s = sc / NCH, c = sc % NCH;
            if (s0 + s < nsk)
                coef[(((long long)k * ncoef + atom * NCH + c) * ldc + s0 + s) * 2 + (i & 1)] =
                    T(ch_scale[atom * NCH + c] * (double)v);
        }
    }
    cluster.sync();  // the other parts keep their shared memory until block 0 has read it
}

// Complex nonlocal scatter, one thread per grid point: Hu[s][g] += sum_e sum_ch conj(P_e,ch) c[a_e, ch][s],
// k-point by k-point (tables zent + k*zstride, states of k at HX + k*ldk). The point's
// first KMAX entries keep their coefficient row in registers, and per k-point their
// Bloch-phase values; the coefficients of a state group are read as {re, im} 16-byte
// pairs (broadcasts across the warp). Entries past KMAX are read from memory in the
// same order.
template <typename T> struct Pair2;
template <> struct Pair2<double> { using type = double2; };
template <> struct Pair2<float> { using type = float2; };

template <typename T, int SG, int NCH, int KMAX>
__global__ void __launch_bounds__(256, 2) k_scatter_all_z(T* __restrict__ HX, long long ldhx, long long ldk,
                                                       long long hxim, int nk, int nsk, long long N,
                                                       const int* __restrict__ row, const int* __restrict__ ent_atom,
                                                       const T* __restrict__ zent, long long zstride,
                                                       const T* __restrict__ coef, int ncoef, long long ldc) {
    using P2 = typename Pair2<T>::type;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N) return;
    const int e0 = row[g], ne = row[g + 1] - e0;
    if (ne == 0) return;
    int cb[KMAX];
#pragma unroll
    for (int kk = 0; kk < KMAX; ++kk) cb[kk] = kk < ne ? __ldg(&ent_atom[e0 + kk]) * NCH : 0;
    for (int k = 0; k < nk; ++k) {
        const T* zk = zent + (long long)k * zstride;
        const P2* ck = reinterpret_cast<const P2*>(coef) + (long long)k * ncoef * ldc;
        T vr[KMAX][NCH], vi[KMAX][NCH];
#pragma unroll
        for (int kk = 0; kk < KMAX; ++kk)
#pragma unroll
            for (int c = 0; c < NCH; ++c) {
                vr[kk][c] = kk < ne ? __ldg(&zk[((long long)(e0 + kk) * NCH + c) * 2]) : T(0);
                vi[kk][c] = kk < ne ? __ldg(&zk[((long long)(e0 + kk) * NCH + c) * 2 + 1]) : T(0);
            }
        for (int s0 = 0; s0 < nsk; s0 += SG) {
            const int gn = min(SG, nsk - s0);
            T accr[SG], acci[SG];
#pragma unroll
            for (int s = 0; s < SG; ++s) accr[s] = acci[s] = T(0);
#pragma unroll
            for (int kk = 0; kk < KMAX; ++kk) {
                if (kk < ne) {
#pragma unroll
                    for (int c = 0; c < NCH; ++c) {
                        const P2* cp = ck + (long long)(cb[kk] + c) * ldc + s0;
#pragma unroll
                        for (int s = 0; s < SG; ++s) {
                            const P2 w = __ldg(cp + s);
                            accr[s] += vr[kk][c] * w.x + vi[kk][c] * w.y;
                            acci[s] += vr[kk][c] * w.y - vi[kk][c] * w.x;
                        }
                    }
                }
            }
            for (int e = e0 + KMAX; e < e0 + ne; ++e) {
                const int base = __ldg(&ent_atom[e]) * NCH;
#pragma unroll
                for (int c = 0; c < NCH; ++c) {
                    const T er = __ldg(&zk[((long long)e * NCH + c) * 2]);
                    const T ei = __ldg(&zk[((long long)e * NCH + c) * 2 + 1]);
                    const P2* cp = ck + (long long)(base + c) * ldc + s0;
#pragma unroll
                    for (int s = 0; s < SG; ++s) {
                        const P2 w = __ldg(cp + s);
                        accr[s] += er * w.x + ei * w.y;
                        acci[s] += er * w.y - ei * w.x;
                    }
                }
            }
            T hr[SG], hi[SG];
            T* hb = HX + (long long)k * ldk + (long long)s0 * ldhx + g;
#pragma unroll
            for (int s = 0; s < SG; ++s) {
                hr[s] = s < gn ? hb[(long long)s * ldhx] : T(0);
                hi[s] = s < gn ? hb[(long long)s * ldhx + hxim] : T(0);
            }
#pragma unroll
            for (int s = 0; s < SG; ++s)
                if (s < gn) {
                    hb[(long long)s * ldhx] = hr[s] + accr[s];
                    hb[(long long)s * ldhx + hxim] = hi[s] + acci[s];
                }
        }
    }
}

// Any-shape fallback for V u - 1/2 (Lap + 2i g.grad - g^2) u at FD order 2, 6 or 8: one
// thread per (point, state), neighbours read from global memory with periodic wrap. The
// sums follow LaplasianKpoint{2nd,6th,8th}_halo_f (order 2: c0 p + cx (p+x + p-x) + ...;
// orders 6, 8: c0 p, then the x, y and z groups).
template <typename T, int ORDER>
__global__ void __launch_bounds__(256) k_kpoint_plain(const HamArgs<T> a) {
    constexpr int R = ORDER == 2 ? 1 : (ORDER == 6 ? 3 : 4);
    const long long N = (long long)a.nx * a.ny * a.nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int s = blockIdx.y;
    const int ix = (int)(i % a.nx), iy = (int)((i / a.nx) % a.ny), iz = (int)(i / ((long long)a.nx * a.ny));
    T c0 = a.c0, dxc[4], dyc[4], dzc[4];
    for (int d = 0; d < 4; ++d) {
        dxc[d] = a.dx[d];
        dyc[d] = a.dy[d];
        dzc[d] = a.dz[d];
    }
    if (a.kco) {
        const T* kc = a.kco + (long long)(s / a.nsk) * 13;
        c0 = kc[0];
        for (int d = 0; d < 4; ++d) {
            dxc[d] = kc[1 + d];
            dyc[d] = kc[5 + d];
            dzc[d] = kc[9 + d];
        }
    }
    T lap[2], der[2], cen[2];
    for (int c = 0; c < 2; ++c) {
        const T* u = a.X + state_offset(a, s, false) + (c ? a.xim : 0);
        auto at = [&](int dx, int dy, int dz) {
            return u[wrap_idx(ix + dx, a.nx) + (long long)a.nx * (wrap_idx(iy + dy, a.ny) + (long long)a.ny * wrap_idx(iz + dz, a.nz))];
        };
        T xm[R], xp[R], ym[R], yp[R], zm[R], zp[R];
        for (int d = 1; d <= R; ++d) {
            xm[d - 1] = at(-d, 0, 0); xp[d - 1] = at(d, 0, 0);
            ym[d - 1] = at(0, -d, 0); yp[d - 1] = at(0, d, 0);
            zm[d - 1] = at(0, 0, -d); zp[d - 1] = at(0, 0, d);
        }
        cen[c] = u[i];
        T l, g;
        if constexpr (ORDER == 2) {
            l = c0 * cen[c] + a.cx[0] * (xp[0] + xm[0]) + a.cy[0] * (yp[0] + ym[0]) + a.cz[0] * (zp[0] + zm[0]);
            g = dxc[0] * (xp[0] - xm[0]);
            g += dyc[0] * (yp[0] - ym[0]);
            g += dzc[0] * (zp[0] - zm[0]);
        } else if constexpr (ORDER == 6) {
            l = c0 * cen[c];
            l += a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
            l += a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
            l += a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
            g = dxc[2] * (xp[2] - xm[2]) + dxc[1] * (xp[1] - xm[1]) + dxc[0] * (xp[0] - xm[0]);
            g += dyc[2] * (yp[2] - ym[2]) + dyc[1] * (yp[1] - ym[1]) + dyc[0] * (yp[0] - ym[0]);
            g += dzc[2] * (zp[2] - zm[2]) + dzc[1] * (zp[1] - zm[1]) + dzc[0] * (zp[0] - zm[0]);
        } else {
            l = c0 * cen[c];
            l += a.cx[3] * (xp[3] + xm[3]) + a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
            l += a.cy[3] * (yp[3] + ym[3]) + a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
            l += a.cz[3] * (zp[3] + zm[3]) + a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
            g = dxc[3] * (xp[3] - xm[3]) + dxc[2] * (xp[2] - xm[2]) + dxc[1] * (xp[1] - xm[1]) + dxc[0] * (xp[0] - xm[0]);
            g += dyc[3] * (yp[3] - ym[3]) + dyc[2] * (yp[2] - ym[2]) + dyc[1] * (yp[1] - ym[1]) + dyc[0] * (yp[0] - ym[0]);
            g += dzc[3] * (zp[3] - zm[3]) + dzc[2] * (zp[2] - zm[2]) + dzc[1] * (zp[1] - zm[1]) + dzc[0] * (zp[0] - zm[0]);
        }
        lap[c] = l;
        der[c] = g;
    }
    const T v = a.V[i];
    T* h = a.HX + state_offset(a, s, true) + i;
    h[0] = (v * cen[0] + lap[0]) - der[1];
    h[a.hxim] = (v * cen[1] + lap[1]) + der[0];
}

template <typename T, int NCH>
int launch_project_z_nch(const DevProjectors& pj, const T* ztab, int nk, int nsk, const T* X, long long ldx,
                         long long ldk, long long xim, T* coef, int forced_sb, int forced_parts, cudaStream_t st) {
    // states per block: the largest of 4 / 2 / 1 (within the register budget of NCH
    // channels) that still gives one block per SM
    constexpr int kMaxSb = NCH <= 4 ? 4 : (NCH == 8 ? 2 : 1);
    const long long zstride = 2LL * pj.nch * pj.npts;
    const long long ldc = coef_ld(nsk);
    const int parts = project_parts(pj, forced_parts);
    int sb = 1;
    if (forced_sb > 0) {
        sb = std::min(forced_sb, kMaxSb);
    } else {
        for (int c : {4, 2})
            if (c <= kMaxSb && (long long)pj.na * parts * nk * ((nsk + c - 1) / c) >= 148) {
                sb = c;
                break;
            }
    }
    const int groups = (nsk + sb - 1) / sb;
    const dim3 g(pj.na * parts, nk * groups);
    cudaError_t e;
#define QG_PROJECT_Z(SBV)                                                                                         \
    e = launch_clustered(k_project_z<T, SBV, NCH>, g, dim3(256), parts, 0, st, X, ldx, ldk, xim, nsk, groups,    \
                         pj.atom_off, pj.pt_g, ztab, zstride, pj.npts, pj.ch_scale, coef, pj.na * NCH, ldc, parts)
    if (sb == 4) {
        if constexpr (kMaxSb >= 4) QG_PROJECT_Z(4);
    } else if (sb == 2) {
        if constexpr (kMaxSb >= 2) QG_PROJECT_Z(2);
    } else {
        QG_PROJECT_Z(1);
    }
#undef QG_PROJECT_Z
    QG_CUDA_TRY(e);
    return QG_OK;
}

template <typename T, int NCH>
void launch_scatter_z_nch(const DevProjectors& pj, const T* zent, int nk, int nsk, T* HX, long long ldhx,
                          long long ldk, long long hxim, long long N, const T* coef, cudaStream_t st) {
    constexpr int KMAX = NCH <= 4 ? 3 : (NCH == 8 ? 2 : 1);
    k_scatter_all_z<T, 4, NCH, KMAX><<<(unsigned)((N + 255) / 256), 256, 0, st>>>(
        HX, ldhx, ldk, hxim, nk, nsk, N, pj.row, pj.ent_atom, zent, 2LL * pj.nch * pj.nent, coef, pj.na * NCH,
        coef_ld(nsk));
}

// Bloch-phase tables for the k-vectors kv (3 per k-point), rebuilt when they change;
// one set per element type (FP64, and FP32 for complex64 states).
template <typename T>
struct ZSet {
    T*& tab;
    T*& ent;
    std::vector<double>& k;
    int& cap;
    bool& ready;
};
ZSet<double> zset(DevProjectors& pj, const double*) { return {pj.ztab, pj.zent, pj.zk, pj.zcap, pj.zready}; }
ZSet<float> zset(DevProjectors& pj, const float*) { return {pj.ztab_f, pj.zent_f, pj.zk_f, pj.zcap_f, pj.zready_f}; }

template <typename T>
int ensure_bloch_tables(qg_hamiltonian h, int nk, const double* kv, cudaStream_t st) {
    DevProjectors& pj = h->pj;
    if (pj.na <= 0 || pj.nch <= 0) return QG_OK;
    ZSet<T> z = zset(pj, static_cast<const T*>(nullptr));
    if (z.ready && (int)z.k.size() == 3 * nk && std::equal(kv, kv + 3 * nk, z.k.begin())) return QG_OK;
    const size_t tab = (size_t)2 * pj.nch * pj.npts, ent = (size_t)2 * pj.nch * pj.nent;
    if (nk > z.cap) {
        cudaFree(z.tab);
        cudaFree(z.ent);
        z.tab = z.ent = nullptr;
        z.cap = 0;
        z.ready = false;
        QG_CUDA_TRY(cudaMalloc(&z.tab, tab * nk * sizeof(T)));
        QG_CUDA_TRY(cudaMalloc(&z.ent, ent * nk * sizeof(T)));
        z.cap = nk;
    }
    const long long total = pj.npts + pj.nent;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    for (int k = 0; k < nk; ++k)
        k_bloch_tables<T><<<blocks, 256, 0, st>>>(pj.tab_d, pj.pt_u, pj.npts, pj.ent_pt, pj.nent, pj.nch,
                                                  kv[3 * k] * h->hx, kv[3 * k + 1] * h->hy, kv[3 * k + 2] * h->hz,
                                                  z.tab + tab * k, z.ent + ent * k);
    QG_CUDA_TRY(cudaGetLastError());
    z.k.assign(kv, kv + 3 * nk);
    z.ready = true;
    return QG_OK;
}

// c0 and the first-derivative coefficients of -1/2 (Lap + 2i g.grad - g^2) at FD order
// 2, 6 or 8, exactly as LaplasianKpoint{2nd,6th,8th}_halo_f form them
// (GridDifferenceKpoint2nd.h:19-35, 6th.h:19-47, 8th.h:18-50): out[0] = c0,
// out[1..4] = dx, [5..8] = dy, [9..12] = dz (first R entries of each used).
void kpoint_coefs(const qg_hamiltonian h, const double* g, double* out) {
    const double coefk = -0.5;
    const double hh[3] = {h->hx, h->hy, h->hz};
    const double gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (h->order == 2)
        out[0] = -coefk * (2.0 / (hh[0] * hh[0]) + 2.0 / (hh[1] * hh[1]) + 2.0 / (hh[2] * hh[2])) - coefk * gg;
    else if (h->order == 6)
        out[0] = -245.0 * coefk *
                     (1.0 / (90.0 * hh[0] * hh[0]) + 1.0 / (90.0 * hh[1] * hh[1]) + 1.0 / (90.0 * hh[2] * hh[2])) -
                 coefk * gg;
    else
        out[0] = -14350.0 / 5040.0 * coefk * (1.0 / (hh[0] * hh[0]) + 1.0 / (hh[1] * hh[1]) + 1.0 / (hh[2] * hh[2])) -
                 coefk * gg;
    const double coef2 = coefk * 2.0;
    for (int d = 0; d < 3; ++d) {
        const bool on = std::fabs(g[d]) >= 1.0e-8;  // the reference's _ddm skips |g| < 1e-8
        double* o = out + 1 + 4 * d;
        o[0] = o[1] = o[2] = o[3] = 0.0;
        if (!on) continue;
        if (h->order == 2) {
            o[0] = coef2 * g[d] / (2.0 * hh[d]);
        } else if (h->order == 6) {
            o[0] = 45.0 * coef2 * g[d] / (60.0 * hh[d]);
            o[1] = -9.0 * coef2 * g[d] / (60.0 * hh[d]);
            o[2] = coef2 * g[d] / (60.0 * hh[d]);
        } else {
            o[0] = 672.0 * coef2 * g[d] / (840.0 * hh[d]);
            o[1] = -168.0 * coef2 * g[d] / (840.0 * hh[d]);
            o[2] = 32.0 * coef2 * g[d] / (840.0 * hh[d]);
            o[3] = -3.0 * coef2 * g[d] / (840.0 * hh[d]);
        }
    }
}

}  // namespace

template <typename T>
int apply_hamiltonian_zk(qg_hamiltonian h, int nk, const double* kv, int nsk, const T* X, long long ldx,
                         long long ldk, T* HX, long long ldhx, long long ldkh, T* coef, cudaStream_t st,
                         PhaseTimer* pt) {
    if (h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    const DevProjectors& pj = h->pj;
    const long long N = h->N();
    HamArgs<T> a{};
    a.X = X; a.ldx = ldx; a.HX = HX; a.ldhx = ldhx; a.ns = nk * nsk;
    a.xim = N; a.hxim = N;
    if constexpr (sizeof(T) == 8) a.V = reinterpret_cast<const T*>(h->V_d);
    else a.V = reinterpret_cast<const T*>(h->V_f);
    a.nx = h->nx; a.ny = h->ny; a.nz = h->nz; a.ty = h->ty;
    a.err = h->ctx->dev_status;
    const double coefk = -0.5;
    const double hh[3] = {h->hx, h->hy, h->hz};
    T* cs[3] = {a.cx, a.cy, a.cz};
    for (int d = 0; d < 3; ++d) {
        if (h->order == 2) {
            cs[d][0] = T(coefk / (hh[d] * hh[d]));
        } else if (h->order == 6) {
            const double s = 90.0 * hh[d] * hh[d];
            cs[d][2] = T(coefk / s);
            cs[d][1] = T(-13.5 * coefk / s);
            cs[d][0] = T(135.0 * coefk / s);
        } else {
            const double s = 5040.0 * hh[d] * hh[d];
            cs[d][3] = T(-9.0 * coefk / s);
            cs[d][2] = T(128.0 * coefk / s);
            cs[d][1] = T(-1008.0 * coefk / s);
            cs[d][0] = T(8064.0 * coefk / s);
        }
    }
    std::vector<double> kc((size_t)13 * nk);
    for (int k = 0; k < nk; ++k) kpoint_coefs(h, kv + 3 * k, kc.data() + 13 * k);
    a.c0 = T(kc[0]);
    for (int d = 0; d < 4; ++d) {
        a.dx[d] = T(kc[1 + d]);
        a.dy[d] = T(kc[5 + d]);
        a.dz[d] = T(kc[9 + d]);
    }
    if (nk > 1) {
        std::vector<T> kct(kc.begin(), kc.end());
        QG_TRY(h->kco.reserve(kct.size() * sizeof(T)));
        // the coefficients are read by this launch only; the stream keeps the copy ordered
        QG_CUDA_TRY(cudaMemcpyAsync(h->kco.ptr, kct.data(), kct.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));  // kct is a host temporary
        a.kco = h->kco.as<T>();
        a.nsk = nsk;
        a.ldkx = ldk;
        a.ldkhx = ldkh;
    }
    const bool nonlocal = pj.na > 0 && pj.nch > 0;
    if (pt) pt->mark(0, st);
    const T* ztab = nullptr;
    const T* zent = nullptr;
    if (nonlocal) {
        QG_TRY(ensure_bloch_tables<T>(h, nk, kv, st));
        if constexpr (sizeof(T) == 8) {
            ztab = pj.ztab;
            zent = pj.zent;
        } else {
            ztab = pj.ztab_f;
            zent = pj.zent_f;
        }
        switch (pj.nch) {
            case 4:
                QG_TRY((launch_project_z_nch<T, 4>(pj, ztab, nk, nsk, X, ldx, ldk, N, coef, h->proj_sb,
                                                    h->proj_parts, st)));
                break;
            case 8:
                QG_TRY((launch_project_z_nch<T, 8>(pj, ztab, nk, nsk, X, ldx, ldk, N, coef, h->proj_sb,
                                                    h->proj_parts, st)));
                break;
            case 16:
                QG_TRY((launch_project_z_nch<T, 16>(pj, ztab, nk, nsk, X, ldx, ldk, N, coef, h->proj_sb,
                                                     h->proj_parts, st)));
                break;
            default: return QG_ERR_UNSUPPORTED;
        }
    }
    if (pt) pt->mark(1, st);
    constexpr int PX = 16 / sizeof(T);
    if (h->stencil_variant == 1 || !stencil_tma_ok<T>(a, h->order, 2) || (nk > 1 && (ldk % PX || ldkh % PX))) {
        dim3 g((unsigned)((N + 255) / 256), (unsigned)(nk * nsk));
        switch (h->order) {
            case 2: k_kpoint_plain<T, 2><<<g, 256, 0, st>>>(a); break;
            case 6: k_kpoint_plain<T, 6><<<g, 256, 0, st>>>(a); break;
            default: k_kpoint_plain<T, 8><<<g, 256, 0, st>>>(a); break;
        }
    } else {
        QG_TRY(launch_stencil_tma<T>(a, h->order, st, 2));
    }
    if (pt) pt->mark(2, st);
    if (nonlocal) {
        switch (pj.nch) {
            case 4: launch_scatter_z_nch<T, 4>(pj, zent, nk, nsk, HX, ldhx, ldkh, N, N, coef, st); break;
            case 8: launch_scatter_z_nch<T, 8>(pj, zent, nk, nsk, HX, ldhx, ldkh, N, N, coef, st); break;
            default: launch_scatter_z_nch<T, 16>(pj, zent, nk, nsk, HX, ldhx, ldkh, N, N, coef, st); break;
        }
    }
    if (pt) pt->mark(-1, st);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

template <typename T>
int apply_hamiltonian_z(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx, T* coef,
                        cudaStream_t st, PhaseTimer* pt) {
    const double kv[3] = {h->gx, h->gy, h->gz};
    return apply_hamiltonian_zk<T>(h, 1, kv, ns, X, ldx, 0, HX, ldhx, 0, coef, st, pt);
}

template int apply_hamiltonian_zk<double>(qg_hamiltonian, int, const double*, int, const double*, long long,
                                          long long, double*, long long, long long, double*, cudaStream_t,
                                          PhaseTimer*);
template int apply_hamiltonian_zk<float>(qg_hamiltonian, int, const double*, int, const float*, long long, long long,
                                         float*, long long, long long, float*, cudaStream_t, PhaseTimer*);
template int apply_hamiltonian_z<double>(qg_hamiltonian, int, const double*, long long, double*, long long, double*,
                                         cudaStream_t, PhaseTimer*);
template int apply_hamiltonian_z<float>(qg_hamiltonian, int, const float*, long long, float*, long long, float*,
                                        cudaStream_t, PhaseTimer*);

}  // namespace qg

namespace {

template <typename T>
int apply_z_checked(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx) {
    if (!h || ns < 0 || (ns > 0 && (!X || !HX))) return QG_ERR_INVALID;
    if (ns == 0) return QG_OK;
    const long long N = h->N();
    if (ldx < 2 * N || ldhx < 2 * N) return QG_ERR_INVALID;
    if (h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    T* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems_z(h, 1, ns) * sizeof(T)));
        coef = h->coef.as<T>();
    }
    return qg::apply_hamiltonian_z<T>(h, ns, X, ldx, HX, ldhx, coef, h->ctx->stream);
}

template <typename T>
int apply_zk_checked(qg_hamiltonian h, int nk, const double* kvecs, int nsk, const T* X, long long ldx, long long ldk,
                     T* HX, long long ldhx, long long ldkh) {
    if (!h || nk <= 0 || nsk < 0 || !kvecs || (nsk > 0 && (!X || !HX))) return QG_ERR_INVALID;
    if (nsk == 0) return QG_OK;
    const long long N = h->N();
    if (ldx < 2 * N || ldhx < 2 * N) return QG_ERR_INVALID;
    if (nk > 1 && (ldk < (long long)nsk * ldx || ldkh < (long long)nsk * ldhx)) return QG_ERR_INVALID;
    if (h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    T* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems_z(h, nk, nsk) * sizeof(T)));
        coef = h->coef.as<T>();
    }
    return qg::apply_hamiltonian_zk<T>(h, nk, kvecs, nsk, X, ldx, ldk, HX, ldhx, ldkh, coef, h->ctx->stream);
}

}  // namespace

extern "C" {

int qg_hamiltonian_apply_zk(qg_hamiltonian h, int nk, const double* kvecs, int nsk, const double* X, long long ldx,
                            long long ldk, double* HX, long long ldhx, long long ldkh) {
    return apply_zk_checked<double>(h, nk, kvecs, nsk, X, ldx, ldk, HX, ldhx, ldkh);
}

int qg_hamiltonian_apply_zkf(qg_hamiltonian h, int nk, const double* kvecs, int nsk, const float* X, long long ldx,
                             long long ldk, float* HX, long long ldhx, long long ldkh) {
    return apply_zk_checked<float>(h, nk, kvecs, nsk, X, ldx, ldk, HX, ldhx, ldkh);
}

int qg_hamiltonian_apply_zf(qg_hamiltonian h, int ns, const float* X, long long ldx, float* HX, long long ldhx) {
    return apply_z_checked<float>(h, ns, X, ldx, HX, ldhx);
}

int qg_hamiltonian_apply_z(qg_hamiltonian h, int ns, const double* X, long long ldx, double* HX, long long ldhx) {
    return apply_z_checked(h, ns, X, ldx, HX, ldhx);
}

int qg_hamiltonian_apply_timed_z(qg_hamiltonian h, int ns, const double* X, long long ldx, double* HX,
                                 long long ldhx, float* ms_phases) {
    if (!h || ns <= 0 || !X || !HX || !ms_phases) return QG_ERR_INVALID;
    const long long N = h->N();
    if (ldx < 2 * N || ldhx < 2 * N) return QG_ERR_INVALID;
    if (h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    double* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems_z(h, 1, ns) * sizeof(double)));
        coef = h->coef.as<double>();
    }
    qg::PhaseTimer pt;
    QG_TRY(qg::apply_hamiltonian_z(h, ns, X, ldx, HX, ldhx, coef, h->ctx->stream, &pt));
    pt.totals(ms_phases);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int qg_hamiltonian_apply_host_z(qg_hamiltonian h, int ns, const double* X, double* HX) {
    if (!h || ns < 0 || (ns > 0 && (!X || !HX))) return QG_ERR_INVALID;
    if (ns == 0) return QG_OK;
    const long long N2 = 2 * h->N();
    return qg::host_pipelined_apply(h, ns, N2, X, HX, [&](int nc, const double* xd, double* hd) {
        return apply_z_checked(h, nc, xd, N2, hd, N2);
    });
}

}  // extern "C"
