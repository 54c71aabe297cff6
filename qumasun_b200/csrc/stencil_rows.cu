// FD stencil + local potential, H psi = V psi - 1/2 Lap psi, two grid rows per consumer
// thread (real states, sm_100a).
//
// Same plane ring as k_stencil_tma (producer lane, bulk async copies counted on
// "full" mbarriers, consumer warps releasing stages through "empty" mbarriers, one
// persistent block per SM, work item = (state, y tile, z slab)), with two changes that
// cut the shared-memory traffic per point, the measured co-limiter of the one-plane
// kernel (13 16-byte loads per two points there):
//  * each consumer thread owns PX x-points of TWO adjacent rows: the rows above and
//    below the pair serve both (8 loads for 2 rows instead of 16 at order 8), and each
//    row's centre value is the other row's nearest y neighbour, from registers;
//  * the producer also streams the tile's rows of V into each stage, so V is read from
//    shared memory next to psi instead of from global memory through a register window.
// Per step and thread: 2 centre + 8 x + 8 y + 2 V loads for 4 points (order 8), against
// 14 for 2 points. The z-window of both rows (2R+1 planes each) stays in registers and
// rotates by renaming over an unrolled z-march. The point sums are those of
// Laplasian{2nd,4th,6th,8th}_halo_f (GridDifference2nd.h:1027-1031, 4th.h:528-530,
// 6th.h:425-429, 8th.h:141-145), grouped as in the other ring kernels, so all of them
// give the same bits. Every mbarrier wait is bounded (QG_ERR_TIMEOUT in the device
// status word on expiry; the block winds down and waits, bounded, for its copies).
#include <cstdint>

#include "qg_internal.h"
#include "stencil_common.cuh"
#include "tma_ring.cuh"

namespace qg {
namespace {

using namespace ring;

constexpr int kRowsThreads = 352;    // one producer warp + up to 320 consumer threads
constexpr int kRowsConsumers = 320;
constexpr size_t kRowsSmemKb = 220;  // ring budget (the V section enlarges each stage)

template <int ORDER>
constexpr int rows_radius() { return ORDER == 2 ? 1 : (ORDER == 8 ? 4 : 3); }

template <typename T>
struct R16;
template <>
struct R16<double> {
    static __device__ __forceinline__ void ld(double (&v)[2], const double* p) {
        const double2 w = *reinterpret_cast<const double2*>(p);
        v[0] = w.x; v[1] = w.y;
    }
    static __device__ __forceinline__ void ldg(double (&v)[2], const double* p) {
        const double2 w = __ldg(reinterpret_cast<const double2*>(p));
        v[0] = w.x; v[1] = w.y;
    }
    static __device__ __forceinline__ void st(double* p, const double (&v)[2]) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    }
};
template <>
struct R16<float> {
    static __device__ __forceinline__ void ld(float (&v)[4], const float* p) {
        const float4 w = *reinterpret_cast<const float4*>(p);
        v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
    }
    static __device__ __forceinline__ void ldg(float (&v)[4], const float* p) {
        const float4 w = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
    }
    static __device__ __forceinline__ void st(float* p, const float (&v)[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};

// -1/2 Lap at one point (same grouping as lap_point of stencil_tma.cu).
template <typename T, int ORDER>
__device__ __forceinline__ T lap_rows(T c, const T* xm, const T* xp, const T* ym, const T* yp, const T* zm,
                                      const T* zp, const HamArgs<T>& a) {
    if constexpr (ORDER == 2) {
        return a.cx[0] * (xp[0] + xm[0] - T(2) * c) + a.cy[0] * (yp[0] + ym[0] - T(2) * c) +
               a.cz[0] * (zp[0] + zm[0] - T(2) * c);
    } else if constexpr (ORDER == 4) {
        return a.cx[2] * ((xp[2] + xm[2]) - T(54) * (xp[1] + xm[1]) + T(783) * (xp[0] + xm[0]) - T(1460) * c) +
               a.cy[2] * ((yp[2] + ym[2]) - T(54) * (yp[1] + ym[1]) + T(783) * (yp[0] + ym[0]) - T(1460) * c) +
               a.cz[2] * ((zp[2] + zm[2]) - T(54) * (zp[1] + zm[1]) + T(783) * (zp[0] + zm[0]) - T(1460) * c);
    } else if constexpr (ORDER == 6) {
        T d = a.c0 * c;
        d += a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
        d += a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
        d += a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
        return d;
    } else {
        T d = a.c0 * c;
        d += a.cx[3] * (xp[3] + xm[3]) + a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
        d += a.cy[3] * (yp[3] + ym[3]) + a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
        d += a.cz[3] * (zp[3] + zm[3]) + a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
        return d;
    }
}

// VR: V rows streamed through the ring (true) or read from global memory one plane ahead
// into registers (false: smaller stages, a deeper ring).
template <typename T, int ORDER, int NXC, bool VR>
__global__ void __launch_bounds__(kRowsThreads, 1) k_stencil_rows(const HamArgs<T> a, const WorkGrid wg, int nst) {
    constexpr int PX = 16 / sizeof(T);
    constexpr int R = rows_radius<ORDER>();
    constexpr int Q = 2 * R + 1;
    constexpr int NV = (R + PX - 1) / PX;
    using VV = R16<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + nst;
    volatile int* ctl = reinterpret_cast<volatile int*>(empty + nst);  // [0] abort, [1] last position issued
    T* ringp = reinterpret_cast<T*>(smem + kBarBytes);

    const int nx = NXC > 0 ? NXC : a.nx, ny = a.ny, nz = a.nz, ty = a.ty;
    const int rows = ty + 2 * R;
    const int psi_elems = rows * nx;
    const int stage_elems = psi_elems + (VR ? ty * nx : 0);  // psi rows, then (VR) the tile's V rows
    const int tpr = nx / PX;
    const int ncons = tpr * (ty / 2);
    const int ncons_warps = (ncons + 31) / 32;
    const int t = threadIdx.x;
    const long long plane = (long long)nx * ny;

    if (t == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], (uint32_t)ncons_warps);
        }
        ctl[0] = 0;
        ctl[1] = -1;
        fence_mbar_init();
    }
    __syncthreads();

    if (t < 32) {
        if (t == 0) produce_planes<T, R, 1, VR>(a, wg, nst, nx, ringp, full, empty, ctl);
    } else if (t < 32 + ncons) {
        const unsigned wmask = __activemask();
        const int lane = t & 31;
        const int c = t - 32;
        const int ix0 = (c % tpr) * PX;
        const int ly0 = 2 * (c / tpr);            // the thread's rows ly0, ly0 + 1 of the tile
        const int cb0 = (R + ly0) * nx + ix0;     // first point of row ly0 inside a stage
        const int vb0 = psi_elems + ly0 * nx + ix0;
        int xo[2 * NV];                           // x-neighbour vectors of row ly0 (row ly0+1: + nx)
#pragma unroll
        for (int v = 0; v < 2 * NV; ++v) {
            const int dv = (v < NV) ? (v - NV) : (v - NV + 1);
            int xx = ix0 + dv * PX;
            xx += (xx < 0) ? nx : 0;
            xx -= (xx >= nx) ? nx : 0;
            xo[v] = (R + ly0) * nx + xx;
        }
        int pos = 0;
        bool bad = false;
        for (int item = blockIdx.x; item < wg.items && !bad; item += gridDim.x) {
            const int slab = item % wg.nslab;
            const int tile = (item / wg.nslab) % wg.tiles;
            const int s = item / (wg.nslab * wg.tiles);
            const int iy0 = tile * ty + ly0;
            const int zs = slab * wg.zslab;
            const int ze = min(nz, zs + wg.zslab);
            const long long col = (long long)iy0 * nx + ix0;

            // z-windows of both rows: plane z - R + d in slot (k + d) % Q at unrolled step k
            T q0[Q][PX], q1[Q][PX];
            int j = pos % nst;
            uint32_t ph = (uint32_t)(pos / nst) & 1u;
            bool w = true;
#pragma unroll
            for (int d = 0; d < 2 * R; ++d) {
                if (w && !mbar_wait(&full[j], ph)) w = false;
                VV::ld(q0[d], ringp + j * stage_elems + cb0);
                VV::ld(q1[d], ringp + j * stage_elems + cb0 + nx);
                if (++j == nst) { j = 0; ph ^= 1u; }
            }
            if (__any_sync(wmask, !w)) {
                bad = true;
                break;
            }
            __syncwarp(wmask);
            int jz = pos % nst;
            if (lane == 0)
                for (int d = 0; d < R; ++d) {  // planes zs-R .. zs-1 live on in registers only
                    mbar_arrive(&empty[jz]);
                    if (++jz == nst) jz = 0;
                }
            jz = (pos + R) % nst;
            int jp = j;  // stage of plane z + R
            uint32_t php = ph;
            T* hcol = a.HX + state_offset(a, s, true) + col;
            const T* vcol = a.V + col;
            T vr0[PX], vr1[PX];  // !VR: V of plane z (rows ly0, ly0 + 1), loaded a step ahead
            if constexpr (!VR) {
                VV::ldg(vr0, vcol + (long long)zs * plane);
                VV::ldg(vr1, vcol + (long long)zs * plane + nx);
            }
            for (int z = zs; z < ze && !bad;) {
#pragma unroll
                for (int k = 0; k < Q; ++k) {
                    if (z >= ze) break;
                    const bool ok = mbar_wait(&full[jp], php);
                    if (__any_sync(wmask, !ok)) {
                        bad = true;
                        break;
                    }
                    const int cs = (k + R) % Q;  // centre slot (plane z)
                    VV::ld(q0[(k + 2 * R) % Q], ringp + jp * stage_elems + cb0);
                    VV::ld(q1[(k + 2 * R) % Q], ringp + jp * stage_elems + cb0 + nx);
                    const T* st = ringp + jz * stage_elems;
                    // rows ly0 - R .. ly0 - 1 and ly0 + 2 .. ly0 + 1 + R (shared by both rows)
                    T ya[R][PX], yb[R][PX];
#pragma unroll
                    for (int d = 1; d <= R; ++d) {
                        VV::ld(ya[d - 1], st + cb0 - d * nx);
                        VV::ld(yb[d - 1], st + cb0 + (1 + d) * nx);
                    }
                    T vv0[PX], vv1[PX], vn0[PX], vn1[PX];
                    if constexpr (VR) {
                        VV::ld(vv0, st + vb0);
                        VV::ld(vv1, st + vb0 + nx);
                    } else {
#pragma unroll
                        for (int e = 0; e < PX; ++e) {
                            vv0[e] = vr0[e];
                            vv1[e] = vr1[e];
                        }
                        if (z + 1 < ze) {
                            VV::ldg(vn0, vcol + (long long)(z + 1) * plane);
                            VV::ldg(vn1, vcol + (long long)(z + 1) * plane + nx);
                        }
                    }
                    T out0[PX], out1[PX];
#pragma unroll
                    for (int row = 0; row < 2; ++row) {
                        T xv[(2 * NV + 1) * PX];
#pragma unroll
                        for (int v = 0; v < 2 * NV; ++v) {
                            T tv[PX];
                            VV::ld(tv, st + xo[v] + row * nx);
                            const int slot = (v < NV) ? v : v + 1;
#pragma unroll
                            for (int e = 0; e < PX; ++e) xv[slot * PX + e] = tv[e];
                        }
#pragma unroll
                        for (int e = 0; e < PX; ++e) xv[NV * PX + e] = row ? q1[cs][e] : q0[cs][e];
#pragma unroll
                        for (int e = 0; e < PX; ++e) {
                            T xm[R], xp[R], ym[R], yp[R], zm[R], zp[R];
#pragma unroll
                            for (int d = 1; d <= R; ++d) {
                                xm[d - 1] = xv[NV * PX + e - d];
                                xp[d - 1] = xv[NV * PX + e + d];
                                if (row == 0) {
                                    ym[d - 1] = ya[d - 1][e];
                                    yp[d - 1] = d == 1 ? q1[cs][e] : yb[d - 2][e];
                                    zm[d - 1] = q0[(k + R - d) % Q][e];
                                    zp[d - 1] = q0[(k + R + d) % Q][e];
                                } else {
                                    ym[d - 1] = d == 1 ? q0[cs][e] : ya[d - 2][e];
                                    yp[d - 1] = yb[d - 1][e];
                                    zm[d - 1] = q1[(k + R - d) % Q][e];
                                    zp[d - 1] = q1[(k + R + d) % Q][e];
                                }
                            }
                            const T cval = row ? q1[cs][e] : q0[cs][e];
                            const T lap = lap_rows<T, ORDER>(cval, xm, xp, ym, yp, zm, zp, a);
                            if (row == 0) out0[e] = vv0[e] * cval + lap;
                            else out1[e] = vv1[e] * cval + lap;
                        }
                    }
                    __syncwarp(wmask);
                    if (lane == 0) mbar_arrive(&empty[jz]);  // plane z is no longer read
                    VV::st(hcol + (long long)z * plane, out0);
                    VV::st(hcol + (long long)z * plane + nx, out1);
                    if constexpr (!VR) {
                        if (z + 1 < ze) {
#pragma unroll
                            for (int e = 0; e < PX; ++e) {
                                vr0[e] = vn0[e];
                                vr1[e] = vn1[e];
                            }
                        }
                    }
                    ++z;
                    if (++jz == nst) jz = 0;
                    if (++jp == nst) { jp = 0; php ^= 1u; }
                }
            }
            if (bad) break;
            __syncwarp(wmask);
            if (lane == 0)
                for (int d = 0; d < R; ++d) {  // planes ze .. ze+R-1
                    mbar_arrive(&empty[jz]);
                    if (++jz == nst) jz = 0;
                }
            pos += ze - zs + 2 * R;
        }
        if (bad) {
            ctl[0] = 1;
            if (lane == 0) atomicExch(a.err, (int)QG_ERR_TIMEOUT);
        }
    }
    __syncthreads();
    if (t == 0 && ctl[0]) {
        const int last = ctl[1];
        for (int ps = max(0, last - nst + 1); ps <= last; ++ps) mbar_wait(&full[ps % nst], (uint32_t)(ps / nst) & 1u);
    }
}

// Rows per tile: the largest even divisor of ny (<= 32) keeping the consumers (one per
// PX x-points of a row pair) within the limit and the ring within its budget.
template <typename T>
int rows_tile(int nx, int ny, int R, bool vr) {
    constexpr int PX = 16 / sizeof(T);
    int ty = 0;
    for (int t = 2; t <= 32; t += 2) {
        if (ny % t != 0 || (nx / PX) * (t / 2) > kRowsConsumers) continue;
        const size_t stage = (size_t)((vr ? 2 * t : t) + 2 * R) * nx * sizeof(T);
        if (ring_stages(R, stage, 3, kRowsSmemKb) > 0) ty = t;
    }
    return ty;
}

template <typename T, int ORDER, bool VR, int NXC = 0>
int launch_rows_order(const HamArgs<T>& a, cudaStream_t st) {
    constexpr int PX = 16 / sizeof(T);
    constexpr int R = rows_radius<ORDER>();
    if constexpr (NXC == 0) {
        switch (a.nx) {
            case 40: return launch_rows_order<T, ORDER, VR, 40>(a, st);
            case 80: return launch_rows_order<T, ORDER, VR, 80>(a, st);
            case 120: return launch_rows_order<T, ORDER, VR, 120>(a, st);
            default: break;
        }
    }
    const size_t stage = (size_t)((VR ? 2 * a.ty : a.ty) + 2 * R) * a.nx * sizeof(T);
    const int nst = ring_stages(R, stage, 3, kRowsSmemKb);
    if (nst < 0) return QG_ERR_UNSUPPORTED;
    const size_t smem = kBarBytes + (size_t)nst * stage;
    auto kern = k_stencil_rows<T, ORDER, NXC, VR>;
    if (allow_max_dynamic_smem(kern) != cudaSuccess)
        return QG_ERR_UNSUPPORTED;
    const int ncons = (a.nx / PX) * (a.ty / 2);
    const int threads = 32 + ncons;
    if (threads > kRowsThreads) return QG_ERR_UNSUPPORTED;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        return QG_ERR_UNSUPPORTED;
    const int G0 = sm_count() * per_sm;
    WorkGrid wg;
    wg.tiles = a.ny / a.ty;
    const long long base = (long long)a.ns * wg.tiles;
    wg.nslab = 1;
    while (base * wg.nslab < 4LL * G0 && a.nz / (wg.nslab * 2) >= 2 * R) wg.nslab *= 2;
    wg.zslab = (a.nz + wg.nslab - 1) / wg.nslab;
    wg.nslab = (a.nz + wg.zslab - 1) / wg.zslab;
    wg.items = (int)(base * wg.nslab);
    const int G = std::min(G0, wg.items);
    kern<<<G, threads, smem, st>>>(a, wg, nst);
    return QG_OK;
}

}  // namespace

template <typename T>
bool stencil_rows_ok(const HamArgs<T>& a, int order, bool vring) {
    constexpr int PX = 16 / sizeof(T);
    if (order != 2 && order != 4 && order != 6 && order != 8) return false;
    const int R = order == 2 ? 1 : (order == 8 ? 4 : 3);
    if (a.row || a.nsk > 0) return false;
    if (a.nx % PX != 0 || ((uintptr_t)a.X % 16) || ((uintptr_t)a.HX % 16) || ((uintptr_t)a.V % 16) ||
        (a.ldx % PX) || (a.ldhx % PX) || !a.err || a.ny < 2 * R || a.nx < 2 * R || a.nz < 2 * R)
        return false;
    return rows_tile<T>(a.nx, a.ny, R, vring) > 0;
}

template <typename T>
int launch_stencil_rows(const HamArgs<T>& a, int order, cudaStream_t st, bool vring) {
    if (!stencil_rows_ok<T>(a, order, vring)) return QG_ERR_UNSUPPORTED;
    HamArgs<T> b = a;
    const int R = order == 2 ? 1 : (order == 8 ? 4 : 3);
    b.ty = rows_tile<T>(a.nx, a.ny, R, vring);
    if (vring) {
        switch (order) {
            case 2: return launch_rows_order<T, 2, true>(b, st);
            case 4: return launch_rows_order<T, 4, true>(b, st);
            case 6: return launch_rows_order<T, 6, true>(b, st);
            case 8: return launch_rows_order<T, 8, true>(b, st);
            default: return QG_ERR_INVALID;
        }
    }
    switch (order) {
        case 2: return launch_rows_order<T, 2, false>(b, st);
        case 4: return launch_rows_order<T, 4, false>(b, st);
        case 6: return launch_rows_order<T, 6, false>(b, st);
        case 8: return launch_rows_order<T, 8, false>(b, st);
        default: return QG_ERR_INVALID;
    }
}

template bool stencil_rows_ok<double>(const HamArgs<double>&, int, bool);
template bool stencil_rows_ok<float>(const HamArgs<float>&, int, bool);
template int launch_stencil_rows<double>(const HamArgs<double>&, int, cudaStream_t, bool);
template int launch_stencil_rows<float>(const HamArgs<float>&, int, cudaStream_t, bool);

}  // namespace qg
