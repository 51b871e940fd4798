// mDPD pair passes with each pair evaluated once.
//
// k_density_staged: per warp of 32 consecutive particles, the list window of every lane is
//   loaded with all its loads in flight into shared memory (coalesced, locally transposed
//   table), then each lane gathers its neighbours' positions eight at a time.  It computes
//   rho_i (fix_aboundary_rho_meso.cu:119-165) and appends to a second, compact table the
//   entries j within the force cutoff whose source particle is above i, so every pair
//   appears once.
// k_force_half: for each compact entry, the mDPD pair force (pair_mdpd_meso.cu:139-225) is
//   evaluated once; +F goes to i and -F to j through 64-bit fixed-point sums (2^-32 units).
//   Integer addition is associative, so the sums do not depend on the order of the atomics:
//   results are bitwise reproducible, and the pairwise forces cancel exactly (momentum).
// k_finalize: fixed-point sums -> FP32 force (+ body force), final half-kick, sums cleared.
#include "kernels.h"
#include "pair.cuh"

namespace mdpd {

constexpr int kWin = 64;                 // list entries staged per lane per window
constexpr double kFix = 4294967296.0;    // 2^32
constexpr double kFixInv = 1.0 / 4294967296.0;

template <bool HALF>
__global__ void __launch_bounds__(128, 8) k_density_staged(const BoxDesc *__restrict__ boxes,
                                                            const Unit *__restrict__ units, int nunits)
{
    __shared__ int s_idx[4][kWin][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        const int i = U.begin + threadIdx.x;
        const bool live = i < U.end;
        const int c = B.st->cur;
        const bool in_group = live && (B.mask[c][i] & B.rho_bit);
        const int n = live ? B.count[i] : 0;
        int nmax = n;
        for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
        const float4 pi = live ? B.pos[i] : make_float4(0, 0, 0, 0);
        const float h = B.cut_rho, h2 = h * h, rcf2 = B.rc2_force;
        const int ncol = B.n_col, ncol2 = B.n_col2, nlocal = B.nlocal;
        // this lane's row base (locally transposed); i&~31 is the warp's block
        const int *row = B.table + ((U.begin + (w << 5)) & ~31) * ncol + lane;
        int *row2 = B.table2 + (i & ~31) * ncol2 + (i & 31);
        float acc = 0.f;
        int n2 = 0;
        for (int kw = 0; kw < nmax; kw += kWin) {
            const int kend = min(kw + kWin, nmax);
            // stage the window: for a fixed k the 32 lanes read 128 contiguous bytes
#pragma unroll
            for (int k0 = 0; k0 < kWin; k0 += 8) {
                int v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int k = kw + k0 + q;
                    v[q] = k < kend ? __ldcs(row + (k & 31) * ncol + (k & ~31)) : 0;
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) s_idx[w][k0 + q][lane] = v[q];
            }
            __syncwarp();
            const int myend = min(kend, n);
            for (int k0 = kw; k0 < myend; k0 += 8) {
                int j[8];
                float4 pj[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) j[q] = k0 + q < myend ? s_idx[w][k0 + q - kw][lane] : -1;
#pragma unroll
                for (int q = 0; q < 8; ++q) pj[q] = j[q] >= 0 ? __ldg(&B.pos[j[q]]) : make_float4(1e30f, 0, 0, 0);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float dx = pi.x - pj[q].x, dy = pi.y - pj[q].y, dz = pi.z - pj[q].z;
                    const float rsq = dist2(dx, dy, dz);
                    if (rsq < h2 && rsq >= 1e-20f) {
                        const float d = h - rsq * rsqrtf(rsq);  // FP32 rsqrt, as the reference
                        acc = __fmaf_rn(d, d, acc);
                    }
                    if (HALF && rsq < rcf2) {
                        const int jj = j[q];
                        const int src = jj < nlocal ? jj : B.gsrc[jj - nlocal];
                        if (src > i) {  // the pair is evaluated from its lower-index end
                            if (n2 < ncol2) row2[(n2 & 31) * ncol2 + (n2 & ~31)] = jj;
                            ++n2;
                        }
                    }
                }
            }
            __syncwarp();
        }
        if (live) {
            if (HALF) {
                B.count2[i] = min(n2, ncol2);
                if (n2 > ncol2) atomicOr(&B.st->status, kErrList2Overflow);
            }
            if (in_group) {
                const float r = (float)(B.mass[ptype(pi)] * (double)B.rho_factor) * acc;
                B.rho[i] = r;
                if (i >= B.st->n_bulk) {
                    const int g1 = min(B.gfirst[i + 1], B.ghost_cap);
                    for (int g = B.gfirst[i]; g < g1; ++g) B.rho[B.nlocal + g] = r;
                }
            }
        }
    }
}

__device__ __forceinline__ long long to_fix(float v) { return __double2ll_rn((double)v * kFix); }

template <bool EXACT, bool EV, bool UNI>
__global__ void __launch_bounds__(128) k_force_half(const BoxDesc *__restrict__ boxes,
                                                    const Unit *__restrict__ units, int nunits)
{
    __shared__ PairCoeff s_coeff[kMaxTypes * kMaxTypes];
    __shared__ double s_red[4][7];
    int cur_box = -1;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (U.box != cur_box) {
            __syncthreads();
            for (int q = threadIdx.x; q < B.ntype * B.ntype; q += blockDim.x) s_coeff[q] = B.coeff[q];
            cur_box = U.box;
            __syncthreads();
        }
        const int i = U.begin + threadIdx.x;
        const bool live = i < U.end;
        long long fx = 0, fy = 0, fz = 0;
        EvAcc ev = {0, 0, 0, 0, 0, 0, 0};
        if (live) {
            const int ntype = B.ntype, nlocal = B.nlocal;
            const float4 pi = B.pos[i];
            const float4 vi = B.vel[i];
            const uint32_t si = __float_as_uint(vi.w);
            const int ti = ptype(pi);
            const float rho_i = B.rho[i];
            const float dtis = B.dt_inv_sqrt;
            const int n2 = B.count2[i];
            const int ncol2 = B.n_col2;
            const int *row2 = B.table2 + (i & ~31) * ncol2 + (i & 31);
            unsigned long long *fax = B.facc, *fay = B.facc + nlocal, *faz = B.facc + 2 * nlocal;
            int jn = n2 > 0 ? __ldcs(row2) : 0;
            for (int k = 0; k < n2; ++k) {
                const int j = jn;
                const int kn = k + 1;
                jn = kn < n2 ? __ldcs(row2 + (kn & 31) * ncol2 + (kn & ~31)) : 0;
                const float4 pj = __ldg(&B.pos[j]);
                const PairCoeff &cf = s_coeff[UNI ? 0 : ti * ntype + ptype(pj)];
                float px = 0.f, py = 0.f, pz = 0.f;
                pair_term<0, EXACT, EV, false>(B, cf, j, pj, pi, vi, si, rho_i, false, 1.f, 1.f, dtis, px, py, pz, ev);
                const long long qx = to_fix(px), qy = to_fix(py), qz = to_fix(pz);
                fx += qx, fy += qy, fz += qz;
                const int src = j < nlocal ? j : B.gsrc[j - nlocal];
                atomicAdd(fax + src, (unsigned long long)(-qx));
                atomicAdd(fay + src, (unsigned long long)(-qy));
                atomicAdd(faz + src, (unsigned long long)(-qz));
            }
            atomicAdd(fax + i, (unsigned long long)fx);
            atomicAdd(fay + i, (unsigned long long)fy);
            atomicAdd(faz + i, (unsigned long long)fz);
        }
        if (EV) {
            // every pair once, full weight (the reference halves each side's share)
            double vals[7] = {ev.vxx, ev.vyy, ev.vzz, ev.vxy, ev.vxz, ev.vyz, ev.pe};
#pragma unroll
            for (int q = 0; q < 7; ++q)
                for (int o = 16; o > 0; o >>= 1) vals[q] += __shfl_down_sync(0xffffffffu, vals[q], o);
            if ((threadIdx.x & 31) == 0)
                for (int q = 0; q < 7; ++q) s_red[threadIdx.x >> 5][q] = vals[q];
            __syncthreads();
            if (threadIdx.x < 7) {
                double a = 0.0;
                for (int ww = 0; ww < 4; ++ww) a += s_red[ww][threadIdx.x];
                B.partial[(size_t)(U.begin / kUnit) * kPartialStride + 1 + threadIdx.x] = a;
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kUnit) k_finalize(const BoxDesc *__restrict__ boxes,
                                                    const Unit *__restrict__ units, int nunits, int kick)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        const int i = U.begin + threadIdx.x;
        if (i >= U.end) continue;
        const int c = B.st->cur, n = B.nlocal;
        unsigned long long *fa = B.facc;
        float fx = (float)((double)(long long)fa[i] * kFixInv);
        float fy = (float)((double)(long long)fa[n + i] * kFixInv);
        float fz = (float)((double)(long long)fa[2 * n + i] * kFixInv);
        fa[i] = 0ull, fa[n + i] = 0ull, fa[2 * n + i] = 0ull;
        const int m = B.mask[c][i];
        if (m & B.body_bit) {
            fx += B.body[0];
            fy += B.body[1];
            fz += B.body[2];
        }
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&B.st->status, kErrNonFinite);
        B.f[c][i] = make_float4(fx, fy, fz, 0.f);
        if (kick && (m & B.nve_bit)) {
            const double dtfm = B.dtfm[B.type[c][i] - 1];
            B.v[c][0][i] = __fma_rn(dtfm, (double)fx, B.v[c][0][i]);
            B.v[c][1][i] = __fma_rn(dtfm, (double)fy, B.v[c][1][i]);
            B.v[c][2][i] = __fma_rn(dtfm, (double)fz, B.v[c][2][i]);
        }
    }
}

void launch_density_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c)
{
    const int grid = u.local.n < c.sms * 8 ? (u.local.n > 0 ? u.local.n : 1) : c.sms * 8;
    k_density_staged<true><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
}

void launch_force_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int ev, int kick)
{
    const int grid = u.local.n < c.sms * 16 ? (u.local.n > 0 ? u.local.n : 1) : c.sms * 16;
    if (c.exact_rng) {
        if (ev) k_force_half<true, true, false><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
        else if (c.uniform_types) k_force_half<true, false, true><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
        else k_force_half<true, false, false><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
    } else {
        if (ev) k_force_half<false, true, false><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
        else if (c.uniform_types) k_force_half<false, false, true><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
        else k_force_half<false, false, false><<<grid, 128, 0, s>>>(boxes, u.local.d, u.local.n);
    }
    const int g2 = u.local.n < c.sms * 8 ? (u.local.n > 0 ? u.local.n : 1) : c.sms * 8;
    k_finalize<<<g2, kUnit, 0, s>>>(boxes, u.local.d, u.local.n, kick);
}

}  // namespace mdpd
