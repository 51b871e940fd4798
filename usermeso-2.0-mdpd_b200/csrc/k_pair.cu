// mDPD pair passes with each pair evaluated once.
//
// k_density_rows: one lane per particle row of the full list (32 consecutive particles per
//   warp, the locally transposed table makes each entry index a coalesced warp load), G = 4, 6
//   or 8 neighbour positions in flight per lane (the batch's autotuner picks G). It computes rho_i (fix_aboundary_rho_meso.cu:
//   119-165) and writes, into the particle's row of the compact table, the entries within the
//   force cutoff that the row owns: a local j when j > i, a ghost j when j is an image shifted
//   in the positive direction (kUpperImage in pos.w). The mirrored pair, seen from the other
//   end, has the opposite shift, so every pair is owned by exactly one row. It also writes
//   (x, y, z, rho) of the particle and its ghost images for the force pass's gathers.
// k_force_pairs: the 32 compact rows of a warp are concatenated and split into 32 equal
//   contiguous shares, one per lane (a prefix scan of the row lengths and one binary search),
//   so every lane evaluates the same number of pairs whatever the row lengths. Each entry
//   carries j's type; j's (x, y, z, rho) and velocity/signature are two float4 gathers, loaded
//   for the next pair while the current one is evaluated. The mDPD pair
//   force (pair_mdpd_meso.cu:139-225) is summed for the row in 64-bit fixed point (2^-32
//   units) in registers and flushed when the lane's share moves to the next row; -F goes to
//   j's source particle in the same fixed point, through shared memory when the source is
//   one of the block's 128 rows and global 64-bit atomics otherwise. Integer addition is
//   associative, so no sum depends on the order of the atomics: results are bitwise
//   reproducible and the pairwise forces cancel exactly (total momentum).
// k_finalize: fixed-point sums -> FP32 pair force, final half-kick (body force added in FP64),
//   sums cleared.
#include "kernels.h"
#include "pair.cuh"

namespace mdpd {

// the density pass keeps G neighbour positions in flight per lane (G = 4, 6 or 8, chosen per
// batch by the autotuner; 6 measured fastest on a 4M box); blocks per SM at 64 registers
template <int G> constexpr int density_blocks() { return G <= 4 ? 8 : 7; }
constexpr float kFixF = 4294967296.0f;           // 2^32
constexpr double kFixInv = 1.0 / 4294967296.0;
constexpr float kFixMax = 1.0e9f;                // |F| bound of the fixed-point range (2^63 / 2^32)
constexpr int kEntryTypeShift = 27;              // compact entry: j | (type of j - 1) << 27
constexpr int kEntryIndex = (1 << kEntryTypeShift) - 1;

template <bool HALF, int kGather>
__global__ void __launch_bounds__(128, density_blocks<kGather>()) k_density_rows(const BoxDesc *__restrict__ boxes,
                                                      const Unit *__restrict__ units, int nunits)
{
    const int u = blockIdx.x;
    if (u >= nunits) return;
    const Unit U = units[u];
    const BoxDesc &B = boxes[U.box];
    const int i = U.begin + threadIdx.x;
    const bool live = i < U.end;
    const int c = B.st->cur;
    const bool in_group = live && (B.mask[c][i] & B.rho_bit);
    const int n = live ? MDPD_IDX(B.count[i], B.n_col + 1) : 0;
    int nmax = n;
    for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    const float4 pi = live ? B.pos[i] : make_float4(0, 0, 0, 0);
    const float h = B.cut_rho, h2 = h * h, rcf2 = B.rc2_force;
    const int ncol = B.n_col, nlocal = B.nlocal;
    // unsigned 32-bit offsets: tables of up to 2^32 entries
    const int *row = B.table + ((unsigned)(i & ~31) * (unsigned)ncol + (unsigned)(i & 31));  // entry k at (k & 31) * ncol + (k & ~31)
    const int ncol2 = B.n_col2;
    int *row2 = B.table2 + (size_t)i * ncol2;
    float acc = 0.f;
    int n2 = 0;
    for (int k0 = 0; k0 < nmax; k0 += kGather) {
        int j[kGather];
        float4 pj[kGather];
#pragma unroll
        for (int q = 0; q < kGather; ++q) {
            const int k = k0 + q;
            j[q] = k < n ? MDPD_IDX(__ldcs(row + (k & 31) * ncol + (k & ~31)), n_all(B)) : -1;
        }
#pragma unroll
        for (int q = 0; q < kGather; ++q) pj[q] = j[q] >= 0 ? __ldg(&B.pos[j[q]]) : make_float4(1e30f, 0, 0, 0);
#pragma unroll
        for (int q = 0; q < kGather; ++q) {
            const float dx = pi.x - pj[q].x, dy = pi.y - pj[q].y, dz = pi.z - pj[q].z;
            const float rsq = dist2(dx, dy, dz);
            if (rsq < h2 && rsq >= 1e-20f) {
                const float d = h - rsq * rsqrtf(rsq);  // FP32 rsqrt, as the reference
                acc = __fmaf_rn(d, d, acc);
            }
            if (HALF) {
                const int jj = j[q];
                if (rsq < rcf2 && (jj < nlocal ? jj > i : (pflags(pj[q]) & kUpperImage) != 0)) {
                    if (n2 < ncol2) row2[n2] = jj | (ptype(pj[q]) << kEntryTypeShift);
                    ++n2;
                }
            }
        }
    }
    if (HALF && live) {
        B.count2[i] = min(n2, ncol2);
        if (n2 > ncol2) atomicOr(&B.st->status, kErrList2Overflow);
    }
    if (in_group) {
        const float r = (float)(B.mass[ptype(pi)] * (double)B.rho_factor) * acc;
        B.rho[i] = r;
        if (HALF) B.posrho[i] = make_float4(pi.x, pi.y, pi.z, r);
        if (i >= B.st->n_bulk) {
            const int g1 = min(B.gfirst[i + 1], B.ghost_cap);
            for (int g = B.gfirst[i]; g < g1; ++g) {
                B.rho[nlocal + g] = r;
                if (HALF) {
                    const float4 pg = B.pos[nlocal + g];
                    B.posrho[nlocal + g] = make_float4(pg.x, pg.y, pg.z, r);
                }
            }
        }
    }
}

__device__ __forceinline__ long long to_fix(float v) { return __float2ll_rn(v * kFixF); }

// 64-bit fixed-point add into a shared (lo, hi) pair of 32-bit words with native 32-bit
// atomics: the low word's wrap-arounds carry into the high word, so the pair ends as the exact
// 64-bit sum (mod 2^64) whatever the order of the adds
__device__ __forceinline__ void sadd64(unsigned *lo, unsigned *hi, long long q)
{
    const unsigned ql = (unsigned)q, qh = (unsigned)((unsigned long long)q >> 32);
    const unsigned old = atomicAdd(lo, ql);
    atomicAdd(hi, qh + (old + ql < old ? 1u : 0u));
}

// 7 blocks per SM (up to 72 registers, no spill) measured fastest against 6 and 8
template <bool EXACT, bool EV, bool UNI>
__global__ void __launch_bounds__(128, 7) k_force_pairs(const BoxDesc *__restrict__ boxes,
                                                        const Unit *__restrict__ units, int nunits)
{
    __shared__ PairCoeff s_coeff[kMaxTypes * kMaxTypes];
    __shared__ float4 s_pi[128], s_vi[128];
    __shared__ float s_rho[128];
    __shared__ int s_pre[4][33];
    __shared__ unsigned s_lo[3][128], s_hi[3][128];
    __shared__ double s_red[4][7];
    const int u = blockIdx.x;
    if (u >= nunits) return;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, wb = t & ~31;
    const Unit U = units[u];
    const BoxDesc &B = boxes[U.box];
    for (int q = t; q < (UNI ? 1 : B.ntype * B.ntype); q += blockDim.x) s_coeff[q] = B.coeff[q];
    const int i = U.begin + t;
    const bool live = i < U.end;
    int pre = 0;
    if (live) {
        s_pi[t] = B.pos[i];
        s_vi[t] = B.vel[i];
        s_rho[t] = B.rho[i];
        pre = MDPD_IDX(B.count2[i], B.n_col2 + 1);
    }
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) pre += v;
    }
    s_pre[w][lane + 1] = pre;
    if (lane == 0) s_pre[w][0] = 0;
    for (int c = 0; c < 3; ++c) s_lo[c][t] = s_hi[c][t] = 0u;
    __syncthreads();
    const int *P = s_pre[w];
    const int T = P[32];
    const int i0 = U.begin + wb, nlocal = B.nlocal, ntype = B.ntype, ncol2 = B.n_col2;
    const int m0 = (lane * T) >> 5, m1 = ((lane + 1) * T) >> 5;
    const float dtis = B.dt_inv_sqrt;
    unsigned long long *fax = B.facc, *fay = B.facc + nlocal, *faz = B.facc + 2 * nlocal;
    EvAcc ev = {0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    if (m0 < m1) {
        int r = 0;  // the row holding entry m0: the last r with P[r] <= m0
#pragma unroll
        for (int st = 16; st > 0; st >>= 1)
            if (P[r + st] <= m0) r += st;
        int rbeg = P[r], rend = P[r + 1];
        float4 pi = s_pi[wb + r], vi = s_vi[wb + r];
        float rho_i = s_rho[wb + r];
        long long ax = 0, ay = 0, az = 0;
        // j's state for the next entry is loaded while the current pair is evaluated
        const int en = __ldcs(B.table2 + (size_t)(i0 + r) * ncol2 + (m0 - rbeg));
        int jn = MDPD_IDX(en & kEntryIndex, n_all(B)), tn = en >> kEntryTypeShift;
        float4 pjn = __ldg(&B.posrho[jn]), vjn = __ldg(&B.vel[jn]);
        int srcn = jn < nlocal ? jn : MDPD_IDX(__ldg(&B.gsrc[jn - nlocal]), nlocal);
        for (int m = m0; m < m1; ++m) {
            if (m >= rend) {  // the share moves on to the next non-empty row
                sadd64(&s_lo[0][wb + r], &s_hi[0][wb + r], ax);
                sadd64(&s_lo[1][wb + r], &s_hi[1][wb + r], ay);
                sadd64(&s_lo[2][wb + r], &s_hi[2][wb + r], az);
                ax = ay = az = 0;
                do {
                    ++r;
                    rbeg = rend;
                    rend = P[r + 1];
                } while (m >= rend);
                pi = s_pi[wb + r], vi = s_vi[wb + r];
                rho_i = s_rho[wb + r];
            }
            const int src = srcn, tj = tn;
            const float4 pj = pjn, vj = vjn;  // pj.w: rho of j
            if (m + 1 < m1) {
                int rr = r, rb = rbeg, re = rend;  // entry m + 1: row r or a later non-empty row
                while (m + 1 >= re) {
                    ++rr;
                    rb = re;
                    re = P[rr + 1];
                }
                const int e = __ldcs(B.table2 + (size_t)(i0 + rr) * ncol2 + (m + 1 - rb));
                const int jj = MDPD_IDX(e & kEntryIndex, n_all(B));
                tn = e >> kEntryTypeShift;
                pjn = __ldg(&B.posrho[jj]);
                vjn = __ldg(&B.vel[jj]);
                srcn = jj < nlocal ? jj : MDPD_IDX(__ldg(&B.gsrc[jj - nlocal]), nlocal);
            }
            const PairCoeff &cf = s_coeff[UNI ? 0 : ptype(pi) * ntype + tj];
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float rsq = dist2(dx, dy, dz);
            float px = 0.f, py = 0.f, pz = 0.f;
            if (rsq < cf.cutsq && rsq >= 1e-20f)
                pair_core<0, EXACT, EV, false>(cf, dx, dy, dz, rsq, vi, vj, __float_as_uint(vi.w), rho_i, pj.w,
                                               false, 1.f, 1.f, dtis, px, py, pz, ev);
            bad |= !(fabsf(px) < kFixMax && fabsf(py) < kFixMax && fabsf(pz) < kFixMax);
            const long long qx = to_fix(px), qy = to_fix(py), qz = to_fix(pz);
            ax += qx, ay += qy, az += qz;
            const int d = src - U.begin;
            if ((unsigned)d < 128u) {  // one of this block's rows (src < nlocal, so d < U.end - U.begin)
                sadd64(&s_lo[0][d], &s_hi[0][d], -qx);
                sadd64(&s_lo[1][d], &s_hi[1][d], -qy);
                sadd64(&s_lo[2][d], &s_hi[2][d], -qz);
            } else {
                atomicAdd(fax + src, (unsigned long long)(-qx));
                atomicAdd(fay + src, (unsigned long long)(-qy));
                atomicAdd(faz + src, (unsigned long long)(-qz));
            }
        }
        sadd64(&s_lo[0][wb + r], &s_hi[0][wb + r], ax);
        sadd64(&s_lo[1][wb + r], &s_hi[1][wb + r], ay);
        sadd64(&s_lo[2][wb + r], &s_hi[2][wb + r], az);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&B.st->status, kErrNonFinite);
    __syncthreads();
    if (live) {
        atomicAdd(fax + i, ((unsigned long long)s_hi[0][t] << 32) | s_lo[0][t]);
        atomicAdd(fay + i, ((unsigned long long)s_hi[1][t] << 32) | s_lo[1][t]);
        atomicAdd(faz + i, ((unsigned long long)s_hi[2][t] << 32) | s_lo[2][t]);
    }
    if (EV) {
        // every pair once, full weight (the reference halves each side's share)
        double vals[7] = {ev.vxx, ev.vyy, ev.vzz, ev.vxy, ev.vxz, ev.vyz, ev.pe};
#pragma unroll
        for (int q = 0; q < 7; ++q)
            for (int o = 16; o > 0; o >>= 1) vals[q] += __shfl_down_sync(0xffffffffu, vals[q], o);
        if (lane == 0)
            for (int q = 0; q < 7; ++q) s_red[w][q] = vals[q];
        __syncthreads();
        if (t < 7) {
            double a = 0.0;
            for (int ww = 0; ww < 4; ++ww) a += s_red[ww][t];
            B.partial[(size_t)(U.begin / kUnit) * kPartialStride + 1 + t] = a;
        }
    }
}

__global__ void __launch_bounds__(kUnit) k_finalize(const BoxDesc *__restrict__ boxes,
                                                    const Unit *__restrict__ units, int nunits, int kick)
{
    const int u = blockIdx.x;  // one unit per block: every load of the pass in flight at once
    if (u >= nunits) return;
    {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        const int i = U.begin + threadIdx.x;
        if (i >= U.end) return;
        const int c = B.st->cur, n = B.nlocal;
        unsigned long long *fa = B.facc;
        // every load of the particle is issued before the first store (the compiler may not move
        // a load above a store to a possibly aliased array): one memory round trip, not four
        const long long ax = (long long)fa[i], ay = (long long)fa[n + i], az = (long long)fa[2 * n + i];
        const int m = B.mask[c][i], t = B.type[c][i];
        const double vx = B.v[c][0][i], vy = B.v[c][1][i], vz = B.v[c][2][i];
        const double dtfm = B.dtfm[t - 1];
        const float fx = (float)((double)ax * kFixInv);
        const float fy = (float)((double)ay * kFixInv);
        const float fz = (float)((double)az * kFixInv);
        fa[i] = 0ull, fa[n + i] = 0ull, fa[2 * n + i] = 0ull;
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&B.st->status, kErrNonFinite);
        B.f[c][i] = make_float4(fx, fy, fz, 0.f);  // the pair force; the body force is in the kicks
        if (kick && (m & B.nve_bit)) {
            const bool body = m & B.body_bit;
            B.v[c][0][i] = __fma_rn(dtfm, (double)fx + (body ? B.body[0] : 0.0), vx);
            B.v[c][1][i] = __fma_rn(dtfm, (double)fy + (body ? B.body[1] : 0.0), vy);
            B.v[c][2][i] = __fma_rn(dtfm, (double)fz + (body ? B.body[2] : 0.0), vz);
        }
    }
}

void launch_density_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c)
{
    const int g = u.local.n;
    if (g <= 0) return;
    switch (c.gather) {
    case 4: k_density_rows<true, 4><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
    case 8: k_density_rows<true, 8><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
    default: k_density_rows<true, 6><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
    }
}

void launch_force_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int ev, int kick)
{
    const int g = u.local.n;
    if (g <= 0) return;
    if (c.exact_rng) {
        if (ev) k_force_pairs<true, true, false><<<g, 128, 0, s>>>(boxes, u.local.d, g);
        else if (c.uniform_types) k_force_pairs<true, false, true><<<g, 128, 0, s>>>(boxes, u.local.d, g);
        else k_force_pairs<true, false, false><<<g, 128, 0, s>>>(boxes, u.local.d, g);
    } else {
        if (ev) k_force_pairs<false, true, false><<<g, 128, 0, s>>>(boxes, u.local.d, g);
        else if (c.uniform_types) k_force_pairs<false, false, true><<<g, 128, 0, s>>>(boxes, u.local.d, g);
        else k_force_pairs<false, false, false><<<g, 128, 0, s>>>(boxes, u.local.d, g);
    }
    k_finalize<<<g, kUnit, 0, s>>>(boxes, u.local.d, g, kick);
}

}  // namespace mdpd
