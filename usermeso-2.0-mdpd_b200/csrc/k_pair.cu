// mDPD pair passes with each pair evaluated once.
//
// k_density_rows: one lane per particle row of the list (32 consecutive particles per warp, the
//   locally transposed table makes each entry index a coalesced warp load), G = 4, 6 or 8
//   neighbour positions in flight per lane (the batch's autotuner picks G).  rho_i
//   (fix_aboundary_rho_meso.cu:119-165) is summed in FP32 with the hardware rsqrt, as the
//   reference forms each term; the reference adds the terms in FP64, which changes rho by about
//   1e-7 of its mean and costs ~13 % of this pass.  The pass also writes, into the particle's
//   row of the compact table, the entries within the force cutoff that the row owns (bit 31 of
//   the list entry, set by the list build: a local j when j > i, a ghost j when j is an image
//   shifted in the positive direction).  The mirrored pair, seen from the other end, has the
//   opposite shift, so every pair is owned by exactly one row.  It also writes (x, y, z, rho) of
//   the particle and its ghost images for the force pass's gathers.
// k_force_pairs: the 32 compact rows of a warp are concatenated and split into 32 equal
//   contiguous shares, one per lane (a prefix scan of the row lengths and one binary search), so
//   every lane evaluates the same number of pairs whatever the row lengths.  The concatenated
//   rows are first staged in shared memory by coalesced loads (consecutive lanes, consecutive
//   entries), so the pair loop's entry reads (each lane in a different row) do not touch 32
//   table lines each.  Each entry carries j's type; j's (x, y, z, rho) and velocity/signature are
//   two float4 gathers, loaded for the next pair while the current one is evaluated.  The mDPD pair force (pair_mdpd_meso.cu:139-225)
//   is summed for the row in 64-bit fixed point (2^-32 units) in registers and flushed when the
//   lane's share moves to the next row; -F goes to j's source particle in the same fixed point,
//   through shared memory when the source is one of the block's 128 rows and global 64-bit
//   atomics otherwise.  Integer addition is associative, so no sum depends on the order of the
//   atomics: results are bitwise reproducible and the pairwise forces cancel exactly (total
//   momentum).  Every pair term is checked against the box's fix_pair_max, which keeps each
//   particle's whole sum inside the fixed-point range; a larger or non-finite term sets the
//   non-finite status.
// k_finalize: fixed-point sums -> FP32 pair force, final half-kick (body force added in FP64),
//   sums cleared.
#include "kernels.h"
#include "pair.cuh"

namespace mdpd {

// the density pass keeps G neighbour positions in flight per lane (G = 4, 6 or 8, chosen per
// batch by the autotuner); blocks per SM: 8 at up to 64 registers (G = 4, 6), 7 at up to 72 (G = 8)
template <int G> constexpr int density_blocks() { return G <= 6 ? 8 : 7; }
constexpr float kFixF = 4294967296.0f;           // 2^32
constexpr double kFixInv = 1.0 / 4294967296.0;
constexpr int kEntryTypeShift = 27;              // compact entry: j | (type of j - 1) << 27
constexpr int kEntryIndex = (1 << kEntryTypeShift) - 1;

// ---------------------------------------------------------------------------------------------
// density pass, global indices
// ---------------------------------------------------------------------------------------------
// approximate 1/sqrt(x), denormal inputs taken as 0 (which gives +inf)
__device__ __forceinline__ float rsqrt_ftz(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One lane per row; the geometry of entries goes two at a time through the two-lane FP32
// instructions.  A term is (h - r)^2 with r = rsq * rsqrt(rsq), formed as t = rsq * rsqrt(rsq) - h
// (one rounding; t is -(h - r) exactly) and min(t, 0)^2: pairs beyond the cutoff add 0, and so
// do the particle's own entry and coincident particles (rsq = 0 gives 0 * inf = NaN, which min()
// drops; a denormal rsq gives inf).  The reference skips rsq < 1e-20; here a normal rsq below 1e-20 (two particles
// closer than 1e-10, whose FP32 coordinates are then both below ~1e-3 in magnitude) would add
// h^2.  Rows are padded to the warp's longest with the particle itself.  Owned entries (bit 31,
// set by the list build) within the force cutoff go to the compact row.
template <int kGather, bool UNI> __device__ __forceinline__ void density_rows(const BoxDesc &B, const Unit &U)
{
    static_assert(kGather % 2 == 0, "entries are taken two at a time");
    const int i = U.begin + threadIdx.x;
    const bool live = i < U.end;
    const int c = B.st->cur;
    const bool in_group = live && (B.mask[c][i] & B.rho_bit);
    const int n = live ? MDPD_IDX(B.count[i], B.n_col + 1) : 0;
    int nmax = n;
    for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    // the warp's rows are one contiguous block of the table (entry k of its 32 rows at 32 k): it
    // is asked into L2 at once, so the entry loads after the first group wait on L2, not on DRAM
    if ((threadIdx.x & 31) == 0 && nmax > 0)
        prefetch_l2_bulk(B.table + (unsigned)(i & ~31) * (unsigned)B.n_col, 128u * (unsigned)nmax);
    const int self = live ? i : U.begin;
    const float4 pi = B.pos[self];
    const float h = B.cut_rho, rcf2 = B.rc2_force;
    const unsigned long long pix = pk2(pi.x, pi.x), piy = pk2(pi.y, pi.y), piz = pk2(pi.z, pi.z);
    const unsigned long long nh = pk2(-h, -h);
    const int ncol = B.n_col, ncol2 = B.n_col2;
    // unsigned 32-bit offsets: tables of up to 2^32 entries
    const int *row = B.table + ((unsigned)(i & ~31) * (unsigned)ncol + (unsigned)(i & 31));  // entry k at 32 k
    int *row2 = B.table2 + (size_t)self * ncol2;
    // one FP32 sum in row order: the terms of entries beyond the cutoff are exact zeros, so a row
    // and its filtered copy (full and reduced lists) give the same rho bit for bit
    float acc = 0.f;
    int n2 = 0;
    for (int k0 = 0; k0 < nmax; k0 += kGather) {
        int e[kGather];
        float4 pj[kGather];
#pragma unroll
        for (int q = 0; q < kGather; ++q) e[q] = k0 + q < n ? __ldcs(row + 32 * (k0 + q)) : self;
#pragma unroll
        for (int q = 0; q < kGather; ++q) pj[q] = __ldg(&B.pos[MDPD_IDX(e[q] & kEntryIndexMask, n_all(B))]);
#pragma unroll
        for (int q = 0; q < kGather; q += 2) {
            const unsigned long long dx = sub2(pix, pk2(pj[q].x, pj[q + 1].x));
            const unsigned long long dy = sub2(piy, pk2(pj[q].y, pj[q + 1].y));
            const unsigned long long dz = sub2(piz, pk2(pj[q].z, pj[q + 1].z));
            const unsigned long long rsq = dist2x2(dx, dy, dz);
            float ra, rb;
            upk2(rsq, ra, rb);
            float ta, tb;
            upk2(fma2(rsq, pk2(rsqrt_ftz(ra), rsqrt_ftz(rb)), nh), ta, tb);
            ta = fminf(ta, 0.f);
            tb = fminf(tb, 0.f);
            acc = __fmaf_rn(ta, ta, acc);
            acc = __fmaf_rn(tb, tb, acc);
#pragma unroll
            for (int h2 = 0; h2 < 2; ++h2) {
                const int eq = e[q + h2];
                if (eq < 0 && (h2 ? rb : ra) < rcf2) {
                    const int j = eq & kEntryIndexMask;
                    row2[min(n2, ncol2 - 1)] = UNI ? j : j | (ptype(pj[q + h2]) << kEntryTypeShift);
                    ++n2;
                }
            }
        }
    }
    if (live) {
        B.count2[i] = min(n2, ncol2);
        if (n2 > ncol2) atomicOr(&B.st->status, kErrList2Overflow);
        // a particle outside the density group keeps its rho (not written, as in the reference),
        // but its packed position is refreshed like every other
        const float r = in_group ? (float)(B.mass[ptype(pi)] * B.rho_factor) * acc : B.rho[i];
        if (in_group) B.rho[i] = r;
        B.posrho[i] = make_float4(pi.x, pi.y, pi.z, r);
        if (i >= B.st->n_bulk) {
            const int g1 = min(B.gfirst[i + 1], B.ghost_cap);
            for (int g = B.gfirst[i]; g < g1; ++g) {
                if (in_group) B.rho[B.nlocal + g] = r;
                const float4 pg = B.pos[B.nlocal + g];
                B.posrho[B.nlocal + g] = make_float4(pg.x, pg.y, pg.z, r);
            }
        }
    }
}

template <int kGather, bool UNI>
__global__ void __launch_bounds__(128, density_blocks<kGather>()) k_density_rows(const BoxDesc *__restrict__ boxes,
                                                      const Unit *__restrict__ units, int nunits)
{
    const int u = blockIdx.x;
    if (u >= nunits) return;
    const Unit U = units[u];
    density_rows<kGather, UNI>(boxes[U.box], U);
}

// ---------------------------------------------------------------------------------------------
// force pass
// ---------------------------------------------------------------------------------------------
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

__device__ __forceinline__ unsigned long long join64(unsigned lo, unsigned hi)
{
    return ((unsigned long long)hi << 32) | lo;
}

// compact entries a warp stages in shared memory: its 32 rows hold ~400 at rho 6.05 (12.6 owned
// force-range pairs each); a warp with more reads them from the table
constexpr int kWarpEntries = 640;

// shared memory of the global-index force pass
struct RowsSmem {
    PairCoeff coeff[kMaxTypes * kMaxTypes];
    float4 pi[128], vi[128];
    float rho[128];
    int pre[4][33];
    unsigned lo[3][128], hi[3][128];
    double red[4][7];
    int ent[4][kWarpEntries];  // each warp's concatenated compact rows (when they fit)
};

// the warp's rows [wb, wb + 32) as one list of T entries split into 32 equal shares; P: prefix
// of the row lengths (P[r] entries before row r, P[32] = T)
__device__ __forceinline__ void warp_prefix(int len, int lane, int *P)
{
    int pre = len;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) pre += v;
    }
    P[lane + 1] = pre;
    if (lane == 0) P[0] = 0;
}

// the row holding entry m of the concatenated rows: the last r with P[r] <= m
__device__ __forceinline__ int row_of(const int *P, int m)
{
    int r = 0;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1)
        if (P[r + st] <= m) r += st;
    return r;
}

template <bool EV>
__device__ __forceinline__ void ev_to_partial(const BoxDesc &B, const Unit &U, const EvAcc &ev, double (*red)[7])
{
    // every pair once, full weight (the reference halves each side's share)
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    double vals[8] = {ev.vxx, ev.vyy, ev.vzz, ev.vxy, ev.vxz, ev.vyz, ev.pe, 0.0};
    const double tot = warp_sum_spread(vals);  // the warp's total of value lane / 4
    if ((lane & 3) == 0 && (lane >> 2) < 7) red[w][lane >> 2] = tot;
    __syncthreads();
    if (t < 7) {
        double a = 0.0;
        for (int ww = 0; ww < 4; ++ww) a += red[ww][t];
        B.partial[(size_t)(U.begin / kUnit) * kPartialStride + 1 + t] = a;
    }
}

template <bool EXACT, bool EV, bool UNI>
__device__ __forceinline__ void force_pairs(const BoxDesc &B, const Unit &U, RowsSmem &S, int stage_cap)
{
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, wb = t & ~31;
    for (int q = t; q < (UNI ? 1 : B.ntype * B.ntype); q += blockDim.x) S.coeff[q] = B.coeff[q];
    const int i = U.begin + t;
    const bool live = i < U.end;
    int len = 0;
    if (live) {
        prefetch_l2(B.table2 + (size_t)i * B.n_col2);  // the row's first 32 entries: one line
        S.pi[t] = B.pos[i];
        S.vi[t] = B.vel[i];
        S.rho[t] = B.rho[i];
        len = MDPD_IDX(B.count2[i], B.n_col2 + 1);
    }
    warp_prefix(len, lane, S.pre[w]);
    for (int c = 0; c < 3; ++c) S.lo[c][t] = S.hi[c][t] = 0u;
    __syncthreads();
    const int *P = S.pre[w];
    const int T = P[32];
    const int i0 = U.begin + wb, nlocal = B.nlocal, ntype = B.ntype, ncol2 = B.n_col2;
    const int m0 = (lane * T) >> 5, m1 = ((lane + 1) * T) >> 5;
    const float dtis = B.dt_inv_sqrt, fix_max = B.fix_pair_max;
    unsigned long long *fax = B.facc, *fay = B.facc + nlocal, *faz = B.facc + 2 * nlocal;
    EvAcc ev = {0, 0, 0, 0, 0, 0, 0};
    bool bad = false;
    // the warp's rows, concatenated, into shared memory: consecutive lanes load consecutive
    // entries (a row's entries are contiguous in the table), so the pair loop's entry reads,
    // one per lane in 32 different rows, come from shared memory instead of 32 table lines
    const bool staged = T <= stage_cap;  // warp-uniform; stage_cap is kWarpEntries, or 0 to read the table
    int *const ent = S.ent[w];
    if (staged) {
        for (int m = lane; m < T; m += 32) {
            const int r = row_of(P, m);
            ent[m] = __ldcs(B.table2 + (size_t)(i0 + r) * ncol2 + (m - P[r]));
        }
        __syncwarp();
    }
    if (m0 < m1) {
        int r = row_of(P, m0);
        int rbeg = P[r], rend = P[r + 1];
        float4 pi = S.pi[wb + r], vi = S.vi[wb + r];
        float rho_i = S.rho[wb + r];
        long long ax = 0, ay = 0, az = 0;
        // j's state for the next entry is loaded while the current pair is evaluated
        const int en = staged ? ent[m0] : __ldcs(B.table2 + (size_t)(i0 + r) * ncol2 + (m0 - rbeg));
        int jn = MDPD_IDX(en & kEntryIndex, n_all(B)), tn = en >> kEntryTypeShift;
        float4 pjn = __ldg(&B.posrho[jn]), vjn = __ldg(&B.vel[jn]);
        int srcn = jn < nlocal ? jn : MDPD_IDX(__ldg(&B.gsrc[jn - nlocal]), nlocal);
        for (int m = m0; m < m1; ++m) {
            if (m >= rend) {  // the share moves on to the next non-empty row
                sadd64(&S.lo[0][wb + r], &S.hi[0][wb + r], ax);
                sadd64(&S.lo[1][wb + r], &S.hi[1][wb + r], ay);
                sadd64(&S.lo[2][wb + r], &S.hi[2][wb + r], az);
                ax = ay = az = 0;
                do {
                    ++r;
                    rbeg = rend;
                    rend = P[r + 1];
                } while (m >= rend);
                pi = S.pi[wb + r], vi = S.vi[wb + r];
                rho_i = S.rho[wb + r];
            }
            const int src = srcn, tj = tn;
            const float4 pj = pjn, vj = vjn;  // pj.w: rho of j
            if (m + 1 < m1) {
                int e;
                if (staged) {
                    e = ent[m + 1];
                } else {
                    int rr = r, rb = rbeg, re = rend;  // entry m + 1: row r or a later non-empty row
                    while (m + 1 >= re) {
                        ++rr;
                        rb = re;
                        re = P[rr + 1];
                    }
                    e = __ldcs(B.table2 + (size_t)(i0 + rr) * ncol2 + (m + 1 - rb));
                }
                const int jj = MDPD_IDX(e & kEntryIndex, n_all(B));
                tn = e >> kEntryTypeShift;
                pjn = __ldg(&B.posrho[jj]);
                vjn = __ldg(&B.vel[jj]);
                srcn = jj < nlocal ? jj : MDPD_IDX(__ldg(&B.gsrc[jj - nlocal]), nlocal);
            }
            const PairCoeff &cf = S.coeff[UNI ? 0 : ptype(pi) * ntype + tj];
            const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            const float rsq = dist2(dx, dy, dz);
            float px = 0.f, py = 0.f, pz = 0.f;
            if (rsq < cf.cutsq && rsq >= 1e-20f)
                pair_core<0, EXACT, EV, false>(cf, dx, dy, dz, rsq, vi, vj, __float_as_uint(vi.w), rho_i, pj.w,
                                               false, 1.f, 1.f, dtis, px, py, pz, ev);
            bad |= !(fabsf(px) < fix_max && fabsf(py) < fix_max && fabsf(pz) < fix_max);
            const long long qx = to_fix(px), qy = to_fix(py), qz = to_fix(pz);
            ax += qx, ay += qy, az += qz;
            const int d = src - U.begin;
            if ((unsigned)d < 128u) {  // one of this block's rows (src < nlocal, so d < U.end - U.begin)
                sadd64(&S.lo[0][d], &S.hi[0][d], -qx);
                sadd64(&S.lo[1][d], &S.hi[1][d], -qy);
                sadd64(&S.lo[2][d], &S.hi[2][d], -qz);
            } else {
                atomicAdd(fax + src, (unsigned long long)(-qx));
                atomicAdd(fay + src, (unsigned long long)(-qy));
                atomicAdd(faz + src, (unsigned long long)(-qz));
            }
        }
        sadd64(&S.lo[0][wb + r], &S.hi[0][wb + r], ax);
        sadd64(&S.lo[1][wb + r], &S.hi[1][wb + r], ay);
        sadd64(&S.lo[2][wb + r], &S.hi[2][wb + r], az);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&B.st->status, kErrNonFinite);
    __syncthreads();
    if (live) {
        atomicAdd(fax + i, join64(S.lo[0][t], S.hi[0][t]));
        atomicAdd(fay + i, join64(S.lo[1][t], S.hi[1][t]));
        atomicAdd(faz + i, join64(S.lo[2][t], S.hi[2][t]));
    }
    if (EV) ev_to_partial<EV>(B, U, ev, S.red);
}

// 7 blocks per SM (up to 72 registers, no spill) measured fastest against 6 and 8
template <bool EXACT, bool EV, bool UNI>
__global__ void __launch_bounds__(128, 7) k_force_pairs(const BoxDesc *__restrict__ boxes,
                                                        const Unit *__restrict__ units, int nunits,
                                                        int stage_cap)
{
    __shared__ RowsSmem S;
    const int u = blockIdx.x;
    if (u >= nunits) return;
    const Unit U = units[u];
    force_pairs<EXACT, EV, UNI>(boxes[U.box], U, S, min(stage_cap, kWarpEntries));
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
    if (c.uniform_types) {
        switch (c.gather) {
        case 4: k_density_rows<4, true><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
        case 8: k_density_rows<8, true><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
        default: k_density_rows<6, true><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
        }
    } else {
        switch (c.gather) {
        case 4: k_density_rows<4, false><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
        case 8: k_density_rows<8, false><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
        default: k_density_rows<6, false><<<g, 128, 0, s>>>(boxes, u.local.d, g); break;
        }
    }
}

template <bool EXACT, bool EV, bool UNI>
static void force_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, int stage_cap)
{
    k_force_pairs<EXACT, EV, UNI><<<u.local.n, 128, 0, s>>>(boxes, u.local.d, u.local.n, stage_cap);
}

void launch_force_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int ev, int kick)
{
    const int g = u.local.n;
    if (g <= 0) return;
    const int cap = c.stage_rows ? kWarpEntries : 0;
    if (c.exact_rng) {
        if (ev) force_half<true, true, false>(s, boxes, u, cap);
        else if (c.uniform_types) force_half<true, false, true>(s, boxes, u, cap);
        else force_half<true, false, false>(s, boxes, u, cap);
    } else {
        if (ev) force_half<false, true, false>(s, boxes, u, cap);
        else if (c.uniform_types) force_half<false, false, true>(s, boxes, u, cap);
        else force_half<false, false, false>(s, boxes, u, cap);
    }
    k_finalize<<<g, kUnit, 0, s>>>(boxes, u.local.d, g, kick);
}

}  // namespace mdpd
