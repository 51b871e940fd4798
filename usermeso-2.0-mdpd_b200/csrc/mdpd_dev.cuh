// Device-side types and helpers of the B200 mDPD/DPD timestep path.
//
// One BoxDesc per simulation box lives in device memory.  Every kernel takes the box
// table plus a list of work units {box, begin, end}, so the same kernels step one box,
// a batch of uneven boxes, or the boxes of a serving loop.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mdpd {

constexpr int kMaxTypes = 8;
constexpr int kUnit = 128;          // particles per work unit (multiple of 32)
constexpr int kClassMax = 512;      // largest bucket the in-warp bucket sort accepts
constexpr int kWarpsPerBlock = 8;


// error bits reported per box (status word), mirrored by MDPD_ERR_* in include/mdpd.h
enum : int {
    kErrListOverflow = 1,   // a particle has more than n_col neighbours
    kErrGhostOverflow = 2,  // more ghost images than the ghost capacity
    kErrBucketOverflow = 4, // a bin or reorder bucket holds more than kClassMax particles
    kErrNonFinite = 8,      // NaN/Inf force
    kErrLost = 16,          // particle outside the box by more than one period
    kErrList2Overflow = 32, // more force-range neighbours than the compact list holds
    kErrIndex = 64,         // check build: an index outside its array (the access was skipped)
};

// bit 31 of a neighbour-list entry: the row's centre owns the pair (j a local above the centre,
// or an upper ghost image); the index is the entry & kEntryIndexMask
constexpr unsigned kOwnedEntry = 0x80000000u;
constexpr int kEntryIndexMask = 0x7FFFFFFF;

struct PairCoeff {  // per type pair; FP32 pair arithmetic
    float cut, cutsq, inv_cut, cut_r, inv_cut_r;
    float A, B, gamma, sigma;  // mdpd: A (attractive), B (repulsive); dpd: A = a0
    float expw;
    float e_cut, e_cut_r;     // energy prefactors 0.5*A*cut, 0.5*B*cut_r
};

struct Unit {
    int box, begin, end;
};

// device-resident per-box scalars, updated by kernels
struct BoxState {
    long long step;        // last completed timestep
    int ago;               // steps since last neighbor build
    int moved;             // some particle moved more than skin/2 (this step)
    int rebuild;           // rebuild decided for this step
    int nghost;
    int n_bulk;            // locals before the first border particle
    int status;            // error bits
    int max_count;         // largest neighbour count at the last build
    long long nbuild;
    int cur;               // live copy of the double-buffered arrays
    int pad;
    // seed_now(sn_seed, sn_step) and seed_now(sn_seed, sn_step - 1), computed once per box by
    // the integrate pass of the step before (valid when sn_ok; a host-written state has sn_ok = 0)
    long long sn_step;
    uint32_t sn_seed, sn;
    int sn_ok;
    uint32_t sn_prev;
};

struct BoxDesc {
    // ---- geometry ----
    double lo[3], hi[3], prd[3], cen[3];
    double binsize[3], bininv[3], coord_inv[3];
    double cutghost, triggersq;
    float rc2_tail;
    int mbin[3], nbin;
    int l1_shift;
    int nlocal, nrow, ghost_cap, n_col;
    int every, delay, check;
    // ---- physics ----
    int style;   // 0 mdpd, 1 dpd
    int ntype;
    int exact_rng;
    PairCoeff coeff[kMaxTypes * kMaxTypes];
    double dtfm[kMaxTypes];  // 0.5*dt*ftm2v * rcp(mass)
    double mass[kMaxTypes];
    double dtv;
    float dt_inv_sqrt;
    uint32_t seed;
    int nve_bit;
    int rho_bit;
    float cut_rho;
    double rho_factor;    // 15/(2 pi cut_rho^5), FP64 as the reference (fix_aboundary_rho_meso.cu:90)
    int body_bit;
    double body[3];       // fix addforce/meso: added in FP64 in both half-kicks (f holds the pair force)
    int arb_bc, mobile_bit, wall_bit;   // wall coupling (pair_style mdpd/meso ... fluid wall)
    int wall_fix;                        // aboundary bounce-back active
    float cut_phi, phi_factor, dw_factor, phi_c;
    double dtf;
    // ---- per-particle arrays (locals), double-buffered for the reorder: the live copy
    //      is [st->cur], the other receives the permuted state at a rebuild ----
    double *x[2][3], *v[2][3], *xh[3];
    float4 *f[2];
    int *tag[2], *type[2], *mask[2];
    // ---- packed FP32 state, locals then ghosts ----
    float4 *pos, *vel;
    float *rho;           // locals then ghosts
    float4 *posrho;       // (x, y, z, rho) of locals then ghosts, written by the pair-once density pass
    float *phi[2];        // wall volume fraction of locals (double-buffered with x)
    int *gsrc, *gimg, *gfirst;
    // ---- neighbour list (transposed per 32 particles: entry k of i at (i&~31)*n_col + 32k + (i&31)) ----
    int *count, *table;
    // entries within the force cutoff whose source index is above the particle's (each pair
    // once), compacted by the density pass for the force pass
    int *count2, *table2;
    int n_col2;
    unsigned long long *facc;  // 3 x nlocal fixed-point force sums (2^-32 units), SoA
    // largest |pair force component| the fixed-point sums accept: 2^31 / (n_col + 1).  A
    // particle's sum has one term per full-list neighbour, at most n_col of them (a longer row
    // is a list overflow), so terms below this bound add to less than 2^31 and the int64 sum in
    // 2^-32 units cannot wrap; a larger term sets the non-finite status
    float fix_pair_max;
    float rc2_force;      // largest force cutoff squared
    // pair-once boxes without walls keep, of the pairs within the list cutoff, only those the
    // passes can use before the next build: the owned ones and those within the density cutoff
    // plus the skin (rn2_list, squared, with a 1e-3 margin over the FP32 rounding of positions)
    float rn2_list;
    int list_reduce;      // set by the batch that steps the box
    // fix aboundary/meso: Gaussian wall density over the wall particles of the list row
    int ab_mobile_bit, ab_wall_bit;
    float ab_rho0, ab_sigma, ab_nfactor;
    // ---- rebuild scratch ----
    int *bin_rank;        // Morton rank of each bin (reorder class order)
    int *cls_count, *cls_start, *cls_cursor;  // 2*nbin
    int *cls_of;          // class of each local
    int *sub_of;          // secondary key of each local
    int *perm;            // new -> old
    int *bin_of;          // bin of locals+ghosts
    int *bin_count, *bin_start, *bin_cursor;  // nbin (+1)
    int *bin_order;       // bin-sorted particle indices
    float4 *bpos;         // positions in bin order
    int *scan_part;       // per-chunk partial sums for scans
    // ---- thermo partials ----
    double *partial;      // per unit thermo partials (kPartialStride doubles)
    BoxState *st;
};

constexpr int kPartialStride = 18;  // see k_thermo_units for the slot map

// ---------------------------------------------------------------------------
// counter-based RNG (TEA, GPU variant of Zafar et al.) and the reference's
// own gaussian transform, restated so the FP64 value is bit-identical.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void tea_core(uint32_t &v0, uint32_t &v1, int rounds)
{
    uint32_t sum = 0;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int r = 0; r < rounds; ++r) {
        sum += 0x9E3779B9u;
        v0 += ((v1 << 4) + 0xA341316Cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xC8013EA4u);
        v1 += ((v0 << 4) + 0xAD90777Du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7E95761Eu);
    }
}

template <int N> __host__ __device__ __forceinline__ uint32_t premix_tea(uint32_t v0, uint32_t v1)
{
    tea_core(v0, v1, N);
    return v0 ^ v1;
}

__host__ __device__ __forceinline__ uint32_t brev32(uint32_t x)
{
#ifdef __CUDA_ARCH__
    return __brev(x);
#else
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) r |= ((x >> i) & 1u) << (31 - i);
    return r;
#endif
}

__host__ __device__ __forceinline__ uint64_t spread3(uint32_t x)
{
    uint64_t r = x & 0x1FFFFFu;
    r = (r | (r << 32)) & 0x1F00000000FFFFull;
    r = (r | (r << 16)) & 0x1F0000FF0000FFull;
    r = (r | (r << 8)) & 0x100F00F00F00F00Full;
    r = (r | (r << 4)) & 0x10C30C30C30C30C3ull;
    r = (r | (r << 2)) & 0x1249249249249249ull;
    return r;
}

__host__ __device__ __forceinline__ uint64_t morton3(uint32_t x, uint32_t y, uint32_t z)
{
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// Rank of bin (x, y, z) among the bins of an mx x my x mz grid ordered by morton3: the bins
// before it are counted octree level by level, from the top.  At level L the bin lies in an
// octant (z bit, y bit, x bit of L) of a cube of side 2^(L+1); every octant of that cube with a
// smaller index comes earlier in Morton order, with all of its bins that lie in the grid.  No
// sort, so a device thread per bin ranks any grid shape.
__host__ __device__ __forceinline__ int morton_rank(int x, int y, int z, int mx, int my, int mz)
{
    int top = 0;
    while ((1 << top) < mx || (1 << top) < my || (1 << top) < mz) ++top;
    long long rank = 0;
    for (int L = top - 1; L >= 0; --L) {
        const int size = 1 << L;
        const int px = (x >> (L + 1)) << (L + 1), py = (y >> (L + 1)) << (L + 1), pz = (z >> (L + 1)) << (L + 1);
        const int mine = (((z >> L) & 1) << 2) | (((y >> L) & 1) << 1) | ((x >> L) & 1);
        for (int c = 0; c < mine; ++c) {
            const int ox = px + (c & 1) * size, oy = py + ((c >> 1) & 1) * size, oz = pz + ((c >> 2) & 1) * size;
            const long long cx = mx - ox < 0 ? 0 : (mx - ox > size ? size : mx - ox);
            const long long cy = my - oy < 0 ? 0 : (my - oy > size ? size : my - oy);
            const long long cz = mz - oz < 0 ? 0 : (mz - oz > size ? size : mz - oz);
            rank += cx * cy * cz;
        }
    }
    return (int)rank;
}

// seed of the current step: premix_TEA<64>(seed, step)
__host__ __device__ __forceinline__ uint32_t seed_now(uint32_t seed, long long step)
{
    return premix_tea<64>(seed, (uint32_t)step);
}

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t sig_mdpd(int tag, uint32_t sn)
{
    return premix_tea<32>(brev32((uint32_t)tag), sn);
}

__device__ __forceinline__ uint32_t sig_dpd(int tag, float vx, float vy, float vz, uint32_t sn)
{
    uint32_t a = (__float_as_uint(vx) & 0x7FF000u) >> 12;
    uint32_t b = (__float_as_uint(vy) & 0x7FF000u) >> 12;
    uint32_t c = (__float_as_uint(vz) & 0x7FF000u) >> 12;
    return sn ^ premix_tea<16>(brev32((uint32_t)tag), (uint32_t)morton3(a, b, c));
}

// reciprocal by magic seed + 4 Newton steps, each step one FMA pair
__host__ __device__ __forceinline__ double rcp_newton(double x)
{
#ifdef __CUDA_ARCH__
    double xinv = __longlong_as_double(0x7FDE62361B1C4042LL - __double_as_longlong(x));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double e = __fma_rn(x, xinv, -1.0);
        xinv = __fma_rn(-e, xinv, xinv);
    }
    return xinv;
#else
    union { double d; long long l; } u;
    u.d = x;
    u.l = 0x7FDE62361B1C4042LL - u.l;
    double xinv = u.d;
    for (int k = 0; k < 4; ++k) {
        double e = __builtin_fma(x, xinv, -1.0);
        xinv = __builtin_fma(-e, xinv, xinv);
    }
    return xinv;
#endif
}

__device__ __forceinline__ double rsqrt_newton(double x)
{
    double r = __longlong_as_double(0x5FE660FCB5422422LL - (__double_as_longlong(x) >> 1));
    double x2m = __dmul_rn(x, -0.5);
#pragma unroll
    for (int k = 0; k < 4; ++k) r = __dmul_rn(r, __fma_rn(__dmul_rn(r, r), x2m, 1.5));
    return r;
}

// log2(x * 2^-32) for x >= 1 with the reference's 8th-order polynomial
__device__ __forceinline__ double log2u_exact(uint32_t x)
{
    int I = 31 - __clz(x);
    double xm = __dmul_rn((double)x, __longlong_as_double((long long)(1023 - I) << 52));
    bool pred = xm > 1.4142135623730950488;
    // the scale into [1/sqrt2, sqrt2) is fused into both x-1 and x+1, as the reference's
    // compiled code does
    const double m = pred ? 0.5 : 7.0710678118654757274E-1;
    double z = __dmul_rn(__fma_rn(xm, m, -1.0), rcp_newton(__fma_rn(xm, m, 1.0)));
    double y = __dmul_rn(__dmul_rn(z, z), 33.9705627484771406);
    double s = 2.55854634203511155E-7;
    s = __fma_rn(s, y, 1.05013262724846015E-5);
    s = __fma_rn(s, y, 5.00072802051539862E-4);
    s = __fma_rn(s, y, 2.83126505877817866E-2);
    s = __fma_rn(s, y, 2.88539008179006374E+0);
    return __fma_rn(z, s, __dadd_rn(pred ? 1.0 : 0.5, (double)(I - 32)));
}

__device__ __forceinline__ double cospi_exact(double x)
{
    x = __fma_rn(2.0, x, -1.0);  // exact: 2x is exact
    double x2 = __dmul_rn(x, x);
    double s = 3.41817283473266926E-6;
    s = __fma_rn(s, x2, -1.60217135750921262E-4);
    s = __fma_rn(s, x2, 4.68162024021793872E-3);
    s = __fma_rn(s, x2, -7.96925872866600517E-2);
    s = __fma_rn(s, x2, 6.45964092644060746E-1);
    s = __fma_rn(s, x2, -1.57079632662144460E+0);
    return __dmul_rn(s, x);
}

// bit-exact FP64 pairwise gaussian from two signatures (symmetric in i,j)
__device__ __forceinline__ double gaussian_exact(uint32_t si, uint32_t sj)
{
    uint32_t v0 = max(si, sj), v1 = min(si, sj);
    tea_core(v0, v1, 4);
    double f = __dmul_rn(cospi_exact(__dmul_rn((double)(v0 & 0x7FFFFFFFu), 4.6566128730773925781E-10)),
                         (v0 & 0x80000000u) ? 1.0 : -1.0);
    double a = __dmul_rn(-2.0 * 6.9314718055994528623E-1, log2u_exact(max(v1, 1u)));
    double r = __dmul_rn(a, rsqrt_newton(a));
    double g = __dmul_rn(r, f);
    return fmax(-4.0, fmin(g, 4.0));
}

// FP32 transform of the same TEA words (same polynomial for the angle; the log of the radius
// word keeps its relative accuracy near 2^32, where the radius is tiny)
__device__ __forceinline__ float gaussian_fast(uint32_t si, uint32_t sj)
{
    uint32_t v0 = max(si, sj), v1 = min(si, sj);
    tea_core(v0, v1, 4);
    // 2u - 1 with u = (v0 & 0x7fffffff) * 2^-31, formed as (w - 2^30) * 2^-30 (one rounding)
    const float x = (float)((int)(v0 & 0x7FFFFFFFu) - (1 << 30)) * 9.3132257461547852e-10f;
    const float x2 = x * x;
    float s = 3.41817283473266926E-6f;
    s = __fmaf_rn(s, x2, -1.60217135750921262E-4f);
    s = __fmaf_rn(s, x2, 4.68162024021793872E-3f);
    s = __fmaf_rn(s, x2, -7.96925872866600517E-2f);
    s = __fmaf_rn(s, x2, 6.45964092644060746E-1f);
    s = __fmaf_rn(s, x2, -1.57079632662144460E+0f);
    const float f = (v0 & 0x80000000u) ? s * x : -s * x;
    const uint32_t w = max(v1, 1u);
    // a = -2 ln(w 2^-32) without a branch. Upper half (w >= 2^31): ln(1 - y) with the exact
    // distance y = (2^32 - w) 2^-32 in (0, 1/2], as 2 atanh(s) = 2 (s + s^3/3 + ... + s^13/13),
    // s = -y / (2 - y) in [-1/3, 0) (truncation below 1e-8); lower half: the hardware log2.
    const float y = (float)(0u - w) * 2.3283064365386963e-10f;
    const float sr = __fdividef(-y, 2.0f - y), t2 = sr * sr;
    float ps = 1.0f / 13.0f;
    ps = __fmaf_rn(ps, t2, 1.0f / 11.0f);
    ps = __fmaf_rn(ps, t2, 1.0f / 9.0f);
    ps = __fmaf_rn(ps, t2, 1.0f / 7.0f);
    ps = __fmaf_rn(ps, t2, 1.0f / 5.0f);
    ps = __fmaf_rn(ps, t2, 1.0f / 3.0f);
    ps = __fmaf_rn(ps, t2, 1.0f);
    const float a_hi = -4.0f * sr * ps;
    const float a_lo = (__log2f((float)w) - 32.0f) * (float)(-2.0 * 6.9314718055994528623E-1);
    const float a = w >= 0x80000000u ? a_hi : a_lo;
    const float r = a * rsqrtf(a);
    return fmaxf(-4.0f, fminf(r * f, 4.0f));
}

// squared distance with the contraction nvcc applies to dx*dx + dy*dy + dz*dz
__device__ __forceinline__ float dist2(float dx, float dy, float dz)
{
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// Asks the memory system to bring [p, p + bytes) into L2 (a hint: no data returns, nothing waits
// on it).  p 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// ---------------------------------------------------------------------------
// Two-lane FP32 arithmetic (sm_100a .f32x2 instructions): one instruction does the same
// operation on two independent values held as one 64-bit register pair; each half rounds
// exactly as the scalar instruction does.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long pk2(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}

__device__ __forceinline__ void upk2(unsigned long long r, float &a, float &b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}

__device__ __forceinline__ unsigned long long sub2(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// a * b + c on both halves, one rounding each
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// dist2 on both halves: fma(dz, dz, fma(dx, dx, dy * dy))
__device__ __forceinline__ unsigned long long dist2x2(unsigned long long dx, unsigned long long dy,
                                                      unsigned long long dz)
{
    return fma2(dz, dz, fma2(dx, dx, mul2(dy, dy)));
}

// Warp sums of N values (N a power of two, 2..32) by recursive halving: at each of log2(N)
// steps lanes pair across bit o (16, 8, ...), each keeps half of its values and adds the
// partner's copy of that half, so a step moves half as many values as the last; a plain
// butterfly over the remaining lane bits ends it.  N - 1 + (5 - log2 N) shuffles instead of
// 5 N.  Returns, in every lane, the warp's total of value (lane >> (5 - log2 N)) & (N - 1).
// The order of the additions is fixed: the same bits on every run.
template <int N> __device__ __forceinline__ double warp_sum_spread(double (&v)[N])
{
    static_assert(N >= 2 && N <= 32 && (N & (N - 1)) == 0, "N: a power of two up to 32");
    const int lane = threadIdx.x & 31;
    int o = 16;
#pragma unroll
    for (int len = N; len > 1; len >>= 1, o >>= 1) {
        const bool upper = lane & o;  // keeps values [len/2, len), renumbered from 0
#pragma unroll
        for (int k = 0; k < len / 2; ++k) {
            const double give = upper ? v[k] : v[k + len / 2];
            const double keep = upper ? v[k + len / 2] : v[k];
            v[k] = keep + __shfl_xor_sync(0xffffffffu, give, o);
        }
    }
    double r = v[0];
#pragma unroll
    for (; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    return r;
}

// ---------------------------------------------------------------------------
// Index checks of the check build (compiled with -DMDPD_CHECK; `build.py --check` writes
// libmdpd_check.so).  MDPD_IDX(i, n) is i when 0 <= i < n; otherwise it sets kErrIndex in the
// status word of the box B in scope and gives 0, an index every array of the box holds, so the
// access stays in bounds and the host reads the error after the step.  Nothing traps.  In the
// normal build MDPD_IDX(i, n) is i and n is not evaluated.  MDPD_IN(i, n) is the same test as
// a condition (always true in the normal build), for a range the caller skips as a whole.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ bool index_ok(long long i, long long n, int *status)
{
    if (i >= 0 && i < n) return true;
#ifdef __CUDA_ARCH__
    atomicOr(status, kErrIndex);
#else
    __atomic_fetch_or(status, kErrIndex, __ATOMIC_RELAXED);
#endif
    return false;
}

__host__ __device__ __forceinline__ int checked_index(long long i, long long n, int *status)
{
    return index_ok(i, n, status) ? (int)i : 0;
}

#ifdef MDPD_CHECK
#define MDPD_IDX(i, n) ::mdpd::checked_index((i), (n), &B.st->status)
#define MDPD_IN(i, n) ::mdpd::index_ok((i), (n), &B.st->status)
#else
#define MDPD_IDX(i, n) (i)
#define MDPD_IN(i, n) true
#endif

// locals plus the ghost images of the last build: the bound of a neighbour index
__host__ __device__ __forceinline__ int n_all(const BoxDesc &B)
{
    return B.nlocal + (B.st->nghost < B.ghost_cap ? B.st->nghost : B.ghost_cap);
}

// entry k of particle i in the locally transposed table: each group of 32 consecutive
// particles owns 32 * n_col entries, entry k of its particles contiguous at 32 k
__device__ __forceinline__ unsigned list_addr(int i, int k, int n_col)
{
    return (unsigned)(i & ~31) * (unsigned)n_col + (unsigned)(32 * k + (i & 31));
}

__device__ __forceinline__ int clamp_bin(int i, int nmax)
{
    return max(0, min(i, nmax - 1));
}

// (x - lo) * inv + 1.0 contracted into one FMA and truncated, as the reference's binning
__device__ __forceinline__ int bin_coord(double x, double lo, double inv)
{
    return (int)__fma_rn(__dsub_rn(x, lo), inv, 1.0);
}

__device__ __forceinline__ int ptype(const float4 &p) { return __float_as_int(p.w) & 0xFF; }
__device__ __forceinline__ int pflags(const float4 &p) { return __float_as_int(p.w) >> 8; }

// pflags bit of a ghost image shifted in the positive direction (image code > 13, i.e. the
// shift (sx, sy, sz) is lexicographically positive in (sz, sy, sx)); the mirror image of a pair
// seen from its other end has the opposite shift
constexpr int kUpperImage = 4;

__device__ __forceinline__ float ghost_w(float w, int code)
{
    return code > 13 ? __int_as_float(__float_as_int(w) | (kUpperImage << 8)) : w;
}

// packed .w word of a position: type-1 in bits 0-7, mobile bit 8, wall bit 9 (bit 10 on ghosts:
// kUpperImage)
__device__ __forceinline__ float pack_w(const BoxDesc &B, int type, int mask)
{
    int w = (type - 1) & 0xFF;
    if (B.arb_bc) {
        if (mask & B.mobile_bit) w |= 1 << 8;
        if (mask & B.wall_bit) w |= 1 << 9;
    }
    return __int_as_float(w);
}

#endif  // __CUDACC__

}  // namespace mdpd
