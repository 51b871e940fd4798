/*
 * CPU oracle for the USER-MESO DPD/mDPD timestep hot path -- TEST INFRASTRUCTURE ONLY.
 * See mdpd_oracle.h for the pins.  Built with -ffp-contract=off: every fused
 * multiply-add below is spelled out with fma()/fmaf() where the reference either
 * calls __fma_rn or where nvcc contracts the reference's expression.
 */
#include "mdpd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ===================================================================== */
/* RNG: TEA words and the reference's own gaussian transform             */
/* ===================================================================== */

/* TEA key schedule of the GPU-TEA generator (math_meso.h:443-447) */
#define TEA_K0 0xA341316Cu
#define TEA_K1 0xC8013EA4u
#define TEA_K2 0xAD90777Du
#define TEA_K3 0x7E95761Eu
#define TEA_DT 0x9E3779B9u

static inline void tea_core(uint32_t *pv0, uint32_t *pv1, int rounds)
{
    /* __TEA_core<N> (math_meso.h:449-456): sum advances by DT before each round */
    uint32_t v0 = *pv0, v1 = *pv1, sum = 0;
    for (int r = 0; r < rounds; ++r) {
        sum += TEA_DT;
        v0 += ((v1 << 4) + TEA_K0) ^ (v1 + sum) ^ ((v1 >> 5) + TEA_K1);
        v1 += ((v0 << 4) + TEA_K2) ^ (v0 + sum) ^ ((v0 >> 5) + TEA_K3);
    }
    *pv0 = v0;
    *pv1 = v1;
}

uint32_t orc_brev(uint32_t x)
{
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) r |= ((x >> i) & 1u) << (31 - i);
    return r;
}

uint32_t orc_premix_tea(uint32_t v0, uint32_t v1, int rounds)
{
    tea_core(&v0, &v1, rounds); /* premix_TEA<N> (math_meso.h:458-463) */
    return v0 ^ v1;
}

uint32_t orc_seed_now(uint32_t seed, int64_t ntimestep)
{
    /* pair_mdpd_meso.cu:295-297: bigint timestep narrowed to uint */
    return orc_premix_tea(seed, (uint32_t)ntimestep, 64);
}

void orc_sig_mdpd(int n, const int32_t *tag, uint32_t seed_now, uint32_t *sig)
{
    for (int i = 0; i < n; ++i) sig[i] = orc_premix_tea(orc_brev((uint32_t)tag[i]), seed_now, 32);
}

static uint64_t bit_space3(uint32_t x)
{
    /* math_meso.h:176-189: spread the low 21 bits three apart */
    uint64_t r = 0;
    for (int i = 0, j = 0; i < 21; ++i, j += 3) r |= ((uint64_t)((x >> i) & 1u)) << j;
    return r;
}

uint64_t orc_morton3(uint32_t x, uint32_t y, uint32_t z)
{
    return bit_space3(x) | (bit_space3(y) << 1) | (bit_space3(z) << 2);
}

static uint32_t f2u(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
}

static float u2f(uint32_t u)
{
    float f;
    memcpy(&f, &u, 4);
    return f;
}

static uint64_t d2ll(double d)
{
    uint64_t u;
    memcpy(&u, &d, 8);
    return u;
}

static double ll2d(uint64_t u)
{
    double d;
    memcpy(&d, &u, 8);
    return d;
}

void orc_sig_dpd(int n, const int32_t *tag, const float *vel4, uint32_t seed_now, uint32_t *sig)
{
    /* atom_vec_meso.cu:164 with __mantissa (math_meso.h:428-434): 11 exponent-adjacent
     * mantissa bits of each FP32 velocity component, Morton-interleaved, low 32 bits */
    for (int i = 0; i < n; ++i) {
        uint32_t a = (f2u(vel4[4 * i + 0]) & 0x7FF000u) >> 12;
        uint32_t b = (f2u(vel4[4 * i + 1]) & 0x7FF000u) >> 12;
        uint32_t c = (f2u(vel4[4 * i + 2]) & 0x7FF000u) >> 12;
        uint32_t m = (uint32_t)orc_morton3(a, b, c);
        sig[i] = seed_now ^ orc_premix_tea(orc_brev((uint32_t)tag[i]), m, 16);
    }
}

double orc_rcp(double x)
{
    /* __rcp (math_meso.h:229-237): magic seed + 4 Newton steps.  nvcc contracts
     * xinv -= e*xinv into one FMA, which is what runs in the reference. */
    double xinv = ll2d(0x7FDE62361B1C4042ULL - d2ll(x));
    for (int k = 0; k < 4; ++k) {
        double e = fma(x, xinv, -1.0);
        xinv = fma(-e, xinv, xinv);
    }
    return xinv;
}

static double ref_rsqrt(double x)
{
    /* __rsqrt (math_meso.h:209-220) */
    double r = ll2d(0x5FE660FCB5422422ULL - (uint64_t)((int64_t)d2ll(x) >> 1));
    double x2m = x * -0.5;
    for (int k = 0; k < 4; ++k) r *= fma(r * r, x2m, 1.5);
    return r;
}

static double pow2i(int n)
{
    return ll2d((uint64_t)(1023 + n) << 52); /* __2_to_n (math_meso.h:203-206) */
}

static double ref_log2u(uint32_t x)
{
    /* __log2u (math_meso.h:392-423): 8th-order polynomial in z=(x-1)/(x+1) */
    static const double c4 = 2.55854634203511155E-7, c3 = 1.05013262724846015E-5,
                        c2 = 5.00072802051539862E-4, c1 = 2.83126505877817866E-2,
                        c0 = 2.88539008179006374E+0;
    int I = 31 - __builtin_clz(x);
    double xm = (double)x * pow2i(-I);
    double ex = (double)(I - 32);
    int pred = xm > 1.4142135623730950488;
    /* x *= m; z = (x-1)*rcp(x+1): nvcc fuses the scale into both uses (pinned against the
     * reference header's device code in tests/golden/ref_device.json) */
    const double m = pred ? 0.5 : 7.0710678118654757274E-1;
    double z = fma(xm, m, -1.0) * orc_rcp(fma(xm, m, 1.0));
    double y = z * z * 33.9705627484771406;
    double s = c4;
    s = fma(s, y, c3);
    s = fma(s, y, c2);
    s = fma(s, y, c1);
    s = fma(s, y, c0);
    return fma(z, s, (pred ? 1.0 : 0.5) + ex);
}

static double ref_cospi(double x)
{
    /* __cospi (math_meso.h:370-390) */
    static const double c5 = 3.41817283473266926E-6, c4 = -1.60217135750921262E-4,
                        c3 = 4.68162024021793872E-3, c2 = -7.96925872866600517E-2,
                        c1 = 6.45964092644060746E-1, c0 = -1.57079632662144460E+0;
    x = 2.0 * x - 1.0;
    double x2 = x * x;
    double s = c5;
    s = fma(s, x2, c4);
    s = fma(s, x2, c3);
    s = fma(s, x2, c2);
    s = fma(s, x2, c1);
    s = fma(s, x2, c0);
    return s * x;
}

double orc_gaussian_tea4(uint32_t si, uint32_t sj)
{
    /* gaussian_TEA<4>(si > sj, si, sj): the larger signature goes first, so the
     * value is symmetric in (i,j) (pair_mdpd_meso.cu:163, math_meso.h:465-473) */
    uint32_t v0 = si > sj ? si : sj;
    uint32_t v1 = si > sj ? sj : si;
    tea_core(&v0, &v1, 4);
    double f = ref_cospi((double)(v0 & 0x7FFFFFFFu) * 4.6566128730773925781E-10) *
               ((v0 & 0x80000000u) ? 1.0 : -1.0);
    double a = -2.0 * 6.9314718055994528623E-1 * ref_log2u(v1 > 1u ? v1 : 1u);
    double r = a * ref_rsqrt(a); /* __sqrtd */
    double g = r * f;
    if (g > 4.0) g = 4.0;
    if (g < -4.0) g = -4.0;
    return g;
}

void orc_gaussian_batch(int n, const uint32_t *si, const uint32_t *sj, double *out)
{
    for (int i = 0; i < n; ++i) out[i] = orc_gaussian_tea4(si[i], sj[i]);
}

/* ===================================================================== */
/* box, bins, keys, ghosts                                               */
/* ===================================================================== */

static int ceil_to(int x, int inc) { return ((x + inc - 1) / inc) * inc; }

void orc_box_setup(orc_box *b, const double lo[3], const double hi[3], double cutforce,
                   double skin, double rho_est, int nlocal)
{
    memset(b, 0, sizeof(*b));
    for (int d = 0; d < 3; ++d) {
        b->lo[d] = lo[d];
        b->hi[d] = hi[d];
        b->prd[d] = hi[d] - lo[d];
        b->cen[d] = 0.5 * (hi[d] + lo[d]); /* dp2sp_merged (atom_vec_mdpd_atomic_meso.cu:180-184) */
    }
    b->skin = skin;
    b->cutneighmax = cutforce + skin; /* neighbor.cpp:258-268 */
    b->cutghost = b->cutneighmax;     /* comm.cpp:413-415 */
    double vol = b->prd[0] * b->prd[1] * b->prd[2];
    double dens = rho_est > 0 ? rho_est : nlocal / vol; /* neighbor_meso.cu:791-801 */
    double e = dens * (4.0 / 3.0 * 3.142 * pow(b->cutneighmax, 3.0));
    e *= 4.0;
    if (e < 32.0) e = 32.0;
    b->expected_neigh_count = e;
    b->n_col = ceil_to((int)e, 32); /* neigh_list_meso.cu:84 */
    double bin_inv_opt = 1.0 / b->cutneighmax;
    for (int d = 0; d < 3; ++d) {
        int nb = (int)(b->prd[d] * bin_inv_opt);
        if (nb < 1) nb = 1;
        b->mbin[d] = nb + 2; /* neighbor_meso.cu:830-838 */
        b->binsize[d] = b->prd[d] / nb;
        b->bininv[d] = 1.0 / b->binsize[d];
    }
    b->rc2_core = (float)pow(b->cutneighmax - skin, 2.0); /* neigh_build_meso.cu:316-317 */
    b->rc2_tail = (float)pow(b->cutneighmax, 2.0);
}

void orc_pbc(const orc_box *b, int n, double *x, double *y, double *z)
{
    double *c[3] = {x, y, z};
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < n; ++i) {
            /* MesoDomain::pbc (domain_meso.cu:58-110) */
            if (c[d][i] < b->lo[d]) c[d][i] += b->prd[d];
            if (c[d][i] >= b->hi[d]) {
                c[d][i] -= b->prd[d];
                if (c[d][i] < b->lo[d]) c[d][i] = b->lo[d];
            }
        }
}

void orc_borderness(const orc_box *b, int n, const double *x, const double *y, const double *z,
                    int *border)
{
    /* one periodic proc per dim: slab 0 = [-BIG, lo+cutghost], slab 1 = [hi-cutghost, BIG]
     * (comm.cpp:585-610), predicate lo <= x <= hi (comm_meso.h pred_border_single) */
    const double *c[3] = {x, y, z};
    for (int i = 0; i < n; ++i) {
        int cnt = 0;
        for (int d = 0; d < 3; ++d) {
            if (c[d][i] <= b->lo[d] + b->cutghost) cnt++;
            if (c[d][i] >= b->hi[d] - b->cutghost) cnt++;
        }
        border[i] = cnt;
    }
}

static int clamp_int(int i, int nmin, int nmax)
{
    /* clamp at [nmin, nmax) (math_meso.h:165-169) */
    if (i > nmax - 1) i = nmax - 1;
    if (i < nmin) i = nmin;
    return i;
}

/* (x - lo) * inv + 1.0, contracted by nvcc into one FMA, truncated to int */
static int bin_coord(double x, double lo, double inv)
{
    return (int)fma(x - lo, inv, 1.0);
}

void orc_reorder_keys(const orc_box *b, int n, const double *x, const double *y, const double *z,
                      uint64_t *key, int *nbits)
{
    /* MesoAtom::sort_local (atom_meso.cu:346-387) + gpu_build_reorder_keypair<1> (:271-311) */
    const int l2_resoln = 16;
    int max_bin = b->mbin[0];
    if (b->mbin[1] > max_bin) max_bin = b->mbin[1];
    if (b->mbin[2] > max_bin) max_bin = b->mbin[2];
    int l1_width = 3 * (int)floor(log2(max_bin * 2.0));
    int l2_width = (int)(3 * log2((double)l2_resoln));
    int l0_shift = l2_width + l1_width;
    int l1_shift = l2_width;
    uint64_t border_mask = 1ULL << l0_shift;
    double coord_inv[3];
    for (int d = 0; d < 3; ++d) coord_inv[d] = l2_resoln * b->bininv[d];
    const double *c[3] = {x, y, z};
    for (int i = 0; i < n; ++i) {
        uint32_t bid[3], sub[3];
        int border = 0;
        for (int d = 0; d < 3; ++d) {
            bid[d] = (uint32_t)clamp_int(bin_coord(c[d][i], b->lo[d], b->bininv[d]), 0, b->mbin[d]);
            /* sub-bin offset omits box lo (a reference quirk); uint (bid-1) widened to double;
             * nvcc contracts x - (bid-1)*binsize into fma(-(bid-1), binsize, x) */
            double off = fma(-(double)(uint32_t)(bid[d] - 1u), b->binsize[d], c[d][i]);
            sub[d] = (uint32_t)clamp_int((int)(off * coord_inv[d]), 0, l2_resoln);
            if (c[d][i] <= b->lo[d] + b->cutghost) border++;
            if (c[d][i] >= b->hi[d] - b->cutghost) border++;
        }
        uint64_t z1 = orc_morton3(bid[0], bid[1], bid[2]);
        uint64_t z2 = orc_morton3(sub[0], sub[1], sub[2]);
        uint64_t k = (z1 << l1_shift) | z2;
        if (border) k |= border_mask;
        key[i] = k;
    }
    if (nbits) *nbits = 1 + l1_width + l2_width;
}

typedef struct { uint64_t k; int32_t i; } kv_t;

static int kv_cmp(const void *a, const void *b)
{
    const kv_t *x = (const kv_t *)a, *y = (const kv_t *)b;
    if (x->k != y->k) return x->k < y->k ? -1 : 1;
    return x->i < y->i ? -1 : (x->i > y->i);
}

void orc_stable_sort_u64(int n, const uint64_t *key, int32_t *perm)
{
    /* a stable LSD radix sort (sort_meso.h:364-443) orders by (key, original index) */
    kv_t *t = (kv_t *)malloc(sizeof(kv_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        t[i].k = key[i];
        t[i].i = i;
    }
    qsort(t, (size_t)n, sizeof(kv_t), kv_cmp);
    for (int i = 0; i < n; ++i) perm[i] = t[i].i;
    free(t);
}

int orc_ghosts(const orc_box *b, int nlocal, int n_bulk, const double *x, const double *y,
               const double *z, int cap, int32_t *src, int32_t *img)
{
    /* MesoComm::borders (comm_meso.cu:42-193) on one periodic proc: for each dim, swap 0
     * sends slab [-BIG, lo+cutghost] shifted by +prd, swap 1 sends [hi-cutghost, BIG]
     * shifted by -prd; both scan [n_bulk, nlocal+nghost at the start of the dim). */
    const double *c[3] = {x, y, z};
    int ng = 0;
    for (int d = 0; d < 3; ++d) {
        int nlast = nlocal + ng;
        for (int side = 0; side < 2; ++side) {
            double lo = side == 0 ? -1e300 : b->hi[d] - b->cutghost;
            double hi = side == 0 ? b->lo[d] + b->cutghost : 1e300;
            int shift = side == 0 ? +1 : -1;
            for (int i = n_bulk; i < nlast; ++i) {
                int s = i < nlocal ? i : src[i - nlocal];
                int im = i < nlocal ? 13 : img[i - nlocal];
                /* coordinate of candidate i in dim d: its own (unshifted in d) */
                int sd = (d == 0 ? im % 3 : d == 1 ? (im / 3) % 3 : im / 9) - 1;
                double cd = c[d][s] + sd * b->prd[d];
                if (cd >= lo && cd <= hi) {
                    if (ng >= cap) return -1;
                    int sx = im % 3 - 1, sy = (im / 3) % 3 - 1, sz = im / 9 - 1;
                    if (d == 0) sx += shift;
                    if (d == 1) sy += shift;
                    if (d == 2) sz += shift;
                    src[ng] = s;
                    img[ng] = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
                    ng++;
                }
            }
        }
    }
    return ng;
}

static void image_xyz(const orc_box *b, const double *x, const double *y, const double *z,
                      int s, int im, double out[3])
{
    int sx = im % 3 - 1, sy = (im / 3) % 3 - 1, sz = im / 9 - 1;
    /* pack_border_vel: x + pbc*prd with pbc in {-1,0,+1} (exact product) */
    out[0] = x[s] + sx * b->prd[0];
    out[1] = y[s] + sy * b->prd[1];
    out[2] = z[s] + sz * b->prd[2];
}

void orc_pack_pos(const orc_box *b, int nlocal, int nghost, const double *x, const double *y,
                  const double *z, const int32_t *type, const int32_t *src, const int32_t *img,
                  float *pos4)
{
    for (int i = 0; i < nlocal + nghost; ++i) {
        double p[3];
        int s = i < nlocal ? i : src[i - nlocal];
        image_xyz(b, x, y, z, s, i < nlocal ? 13 : img[i - nlocal], p);
        pos4[4 * i + 0] = (float)(p[0] - b->cen[0]);
        pos4[4 * i + 1] = (float)(p[1] - b->cen[1]);
        pos4[4 * i + 2] = (float)(p[2] - b->cen[2]);
        pos4[4 * i + 3] = u2f((uint32_t)(type[s] - 1));
    }
}

void orc_bin_ids(const orc_box *b, int nlocal, int nall, const double *x, const double *y,
                 const double *z, uint32_t *bin)
{
    /* gpu_assign_bin_id (neighbor_meso.cu:390-425); x,y,z hold locals then ghosts */
    const double *c[3] = {x, y, z};
    for (int i = 0; i < nall; ++i) {
        int bid[3];
        for (int d = 0; d < 3; ++d) {
            double v = c[d][i];
            bid[d] = clamp_int(bin_coord(v, b->lo[d], b->bininv[d]), 0, b->mbin[d]);
            if (i >= nlocal) bid[d] = v >= b->lo[d] ? (v <= b->hi[d] ? bid[d] : b->mbin[d] - 1) : 0;
        }
        bin[i] = (uint32_t)(bid[0] + b->mbin[0] * (bid[1] + bid[2] * b->mbin[1]));
    }
}

float orc_dr2f(float dx, float dy, float dz)
{
    /* dx*dx + dy*dy + dz*dz as nvcc contracts it: fma(dz,dz, fma(dx,dx, dy*dy)) */
    return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

/* The list a pair-once box keeps (the engine's reduction of the full list above, not a
 * reference algorithm): of row i, the entries owned by i -- a local j > i, or a ghost image
 * shifted in the positive direction (gimg > 13) -- and those within rn2 (squared, the FP32
 * distance of the list test).  Row order is kept.  Row-major tables of ncol columns. */
void orc_reduce_rows(int nlocal, int ncol, const int32_t *count, const int32_t *table,
                     const float *pos4, const int32_t *gimg, float rn2, int32_t *out_count,
                     int32_t *out_table)
{
    for (int i = 0; i < nlocal; ++i) {
        const int32_t *row = table + (size_t)i * ncol;
        int32_t *out = out_table + (size_t)i * ncol;
        int m = 0;
        for (int k = 0; k < count[i]; ++k) {
            const int j = row[k];
            const int owned = j < nlocal ? j > i : gimg[j - nlocal] > 13;
            const float r2 = orc_dr2f(pos4[4 * i] - pos4[4 * j], pos4[4 * i + 1] - pos4[4 * j + 1],
                                      pos4[4 * i + 2] - pos4[4 * j + 2]);
            if (owned || r2 <= rn2) out[m++] = j;
        }
        out_count[i] = m;
    }
}

/* fix aboundary/meso at the end of a step (gpu_aboundary_v2, fix_aboundary_meso.cu:186-281):
 * a particle of the mobile group is projected half a kick and one drift ahead (v + dt/2 f,
 * x + dt v, unit mass as the reference writes it); the Gaussian density of the wall particles
 * of its whole row (count[i] entries: the reference passes dev_pair_count_core, which the list
 * join gpu_join_neigh_list, neigh_build_meso.cu:188-204, sets to core plus skin) is summed at
 * that point; above rho0/2 the parts of v and f along the direction
 * into the wall (minus the normalised density gradient) are removed twice over.  FP32 as the
 * reference; its contracted forms are written as fmaf.  v and f (the total force) in place. */
static float orc_dot3f(float ax, float ay, float az, float bx, float by, float bz)
{
    return fmaf(az, bz, fmaf(ax, bx, ay * by));
}

void orc_aboundary_meso(int nlocal, const float *pos4, const int32_t *mask_all, const int32_t *count,
                        const int32_t *table, int ncol, int mobile_bit, int wall_bit, double rho0, double sigma,
                        double dt, double *vx, double *vy, double *vz, double *fx, double *fy, double *fz)
{
    const float sg = (float)sigma, r0 = (float)rho0, dtf = (float)dt;
    const float nf = (float)(1.0 / sqrt(pow(2 * M_PI, 3.0) * pow(sigma, 3.0))); /* :275 */
    const float hs = (float)(0.5 * (double)dtf);
    const float ex = -0.5f / sg;
    for (int i = 0; i < nlocal; ++i) {
        if (!(mask_all[i] & mobile_bit)) continue;
        const float v0x = (float)vx[i], v0y = (float)vy[i], v0z = (float)vz[i];
        const float f0x = (float)fx[i], f0y = (float)fy[i], f0z = (float)fz[i];
        const float px = fmaf(hs, f0x, v0x), py = fmaf(hs, f0y, v0y), pz = fmaf(hs, f0z, v0z);
        const float cx = fmaf(dtf, px, pos4[4 * i]), cy = fmaf(dtf, py, pos4[4 * i + 1]),
                    cz = fmaf(dtf, pz, pos4[4 * i + 2]);
        float rho = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
        for (int k = 0; k < count[i]; ++k) {
            const int j = table[(size_t)i * ncol + k];
            if (!(mask_all[j] & wall_bit)) continue;
            const float dx = cx - pos4[4 * j], dy = cy - pos4[4 * j + 1], dz = cz - pos4[4 * j + 2];
            const float w = nf * expf(ex * orc_dr2f(dx, dy, dz));
            rho += w;
            const float ws = w / sg;
            gx = fmaf(dx, ws, gx);
            gy = fmaf(dy, ws, gy);
            gz = fmaf(dz, ws, gz);
        }
        if (rho > 0.5f * r0) {
            const float inv = 1.0f / sqrtf(orc_dot3f(gx, gy, gz, gx, gy, gz));
            const float ex_ = -(gx * inv), ey_ = -(gy * inv), ez_ = -(gz * inv);
            const float vd = fmaxf(0.f, orc_dot3f(v0x, v0y, v0z, ex_, ey_, ez_));
            const float fd = fmaxf(0.f, orc_dot3f(f0x, f0y, f0z, ex_, ey_, ez_));
            vx[i] -= (double)(2.f * vd * ex_);
            vy[i] -= (double)(2.f * vd * ey_);
            vz[i] -= (double)(2.f * vd * ez_);
            fx[i] -= (double)(2.f * fd * ex_);
            fy[i] -= (double)(2.f * fd * ey_);
            fz[i] -= (double)(2.f * fd * ez_);
        }
    }
}

typedef struct { uint64_t key; int bin; } stencil_t;

static int stencil_cmp(const void *a, const void *b)
{
    const stencil_t *x = (const stencil_t *)a, *y = (const stencil_t *)b;
    return x->key < y->key ? -1 : (x->key > y->key);
}

/* 27-bin stencil of a bin, sorted by Morton key with +2^31 on ghost-layer bins
 * (gpu_stencil_full_bin_3d, neighbor_meso.cu:685-738) */
static int stencil_of(const orc_box *b, int bx, int by, int bz, int *out)
{
    stencil_t s[27];
    int n = 0;
    for (int k = -1; k <= 1; ++k)
        for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i) {
                int x = bx + i, y = by + j, z = bz + k;
                if (x < 0 || x >= b->mbin[0] || y < 0 || y >= b->mbin[1] || z < 0 ||
                    z >= b->mbin[2])
                    continue;
                s[n].bin = x + b->mbin[0] * (y + z * b->mbin[1]);
                s[n].key = orc_morton3((uint32_t)x, (uint32_t)y, (uint32_t)z);
                if (x == 0 || x == b->mbin[0] - 1 || y == 0 || y == b->mbin[1] - 1 || z == 0 ||
                    z == b->mbin[2] - 1)
                    s[n].key += 0x80000000ULL;
                n++;
            }
    /* the reference bubble-sorts (unstable swaps only on strict >); keys are unique */
    qsort(s, (size_t)n, sizeof(stencil_t), stencil_cmp);
    for (int i = 0; i < n; ++i) out[i] = s[i].bin;
    return n;
}

int orc_build_list(const orc_box *b, int nlocal, int nall, const double *x, const double *y,
                   const double *z, const float *pos4, int32_t *count, int32_t *count_core,
                   int32_t *table)
{
    int nbin = b->mbin[0] * b->mbin[1] * b->mbin[2];
    uint32_t *bin = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nall > 0 ? nall : 1));
    orc_bin_ids(b, nlocal, nall, x, y, z, bin);
    /* stable bin sort -> bin_start (counting sort keeps index order inside a bin) */
    int *start = (int *)calloc((size_t)nbin + 1, sizeof(int));
    int *order = (int *)malloc(sizeof(int) * (size_t)(nall > 0 ? nall : 1));
    for (int i = 0; i < nall; ++i) start[bin[i] + 1]++;
    for (int c = 0; c < nbin; ++c) start[c + 1] += start[c];
    int *fill = (int *)malloc(sizeof(int) * (size_t)nbin);
    memcpy(fill, start, sizeof(int) * (size_t)nbin);
    for (int i = 0; i < nall; ++i) order[fill[bin[i]]++] = i;
    free(fill);
    int overflow = 0;
    const int ncol = b->n_col;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < nlocal; ++i) {
        int bb = (int)bin[i];
        int bx = bb % b->mbin[0], by = (bb / b->mbin[0]) % b->mbin[1],
            bz = bb / (b->mbin[0] * b->mbin[1]);
        int st[27];
        int ns = stencil_of(b, bx, by, bz, st);
        float xi = pos4[4 * i], yi = pos4[4 * i + 1], zi = pos4[4 * i + 2];
        int nc = 0, nk = 0;
        int32_t *row = table + (size_t)i * ncol;
        for (int s = 0; s < ns; ++s)
            for (int p = start[st[s]]; p < start[st[s] + 1]; ++p) {
                int j = order[p];
                float dx = xi - pos4[4 * j], dy = yi - pos4[4 * j + 1], dz = zi - pos4[4 * j + 2];
                float r2 = orc_dr2f(dx, dy, dz);
                if (j == i || !(r2 <= b->rc2_tail)) continue;
                if (nc + nk >= ncol) {
#pragma omp critical
                    if (!overflow) overflow = i + 1;
                    continue;
                }
                if (r2 <= b->rc2_core) row[nc++] = j;
                else row[ncol - 1 - nk++] = j;
            }
        /* join: skin entries follow core entries, read back-to-front (gpu_join_neigh_list) */
        for (int k = 0; k < nk; ++k) row[nc + k] = row[ncol - nk + k];
        count[i] = nc + nk;
        if (count_core) count_core[i] = nc;
    }
    free(bin);
    free(start);
    free(order);
    return overflow;
}

/* ===================================================================== */
/* pair passes                                                           */
/* ===================================================================== */

static int type_of(const float *pos4, int i) { return (int)(f2u(pos4[4 * i + 3]) & 0xFFu); /* low byte: type-1 */ }

void orc_density(int nlocal, const float *pos4, const int32_t *count, const int32_t *table,
                 int n_col, const int32_t *mask, int groupbit, double cut_rho,
                 const double *mass_type, double *rho)
{
    /* fix_aboundary_rho_meso.cu:88-90 (factor) and :119-165 (kernel).  The reference works in
     * FP32 here and so does this restatement, step for step: the coordinate differences, the
     * squared distance (contracted as orc_dr2f), r = rsq * rsqrt(rsq), (h - r)^2; the weight
     * (h - r)^2 * factor is formed in FP64 and rounded to FP32 (r32 wf), and the sum of
     * m_i * wf is FP64.  The reference's rsqrt is the hardware's approximate FP32 reciprocal
     * square root; 1 / sqrtf (correctly rounded) stands in for it, so single terms may differ
     * in their last bits. */
    const double factor = 15.0 / (2.0 * M_PI * cut_rho * cut_rho * cut_rho * cut_rho * cut_rho);
    const float h = (float)cut_rho;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nlocal; ++i) {
        if (!(mask[i] & groupbit)) continue; /* not written, as in the reference */
        const float xi = pos4[4 * i], yi = pos4[4 * i + 1], zi = pos4[4 * i + 2];
        double mi = mass_type[type_of(pos4, i)];
        double r = 0.0;
        for (int k = 0; k < count[i]; ++k) {
            int j = table[(size_t)i * n_col + k];
            const float dx = xi - pos4[4 * j], dy = yi - pos4[4 * j + 1], dz = zi - pos4[4 * j + 2];
            const float rsq = orc_dr2f(dx, dy, dz);
            if (rsq < h * h && rsq >= 1e-20) {
                const float rr = rsq * (1.0f / sqrtf(rsq));
                const float d = h - rr;
                const float wf = (float)((double)(d * d) * factor);
                r += mi * (double)wf;
            }
        }
        rho[i] = r;
    }
}

void orc_aboundary(int nlocal, double *x, double *y, double *z, double *vx, double *vy,
                   double *vz, const double *xa, const double *ya, const double *za,
                   const int32_t *mask, const int32_t *count, const int32_t *table, int n_col,
                   int mobile_bit, int wall_bit, double cut_phi, double rho_wall, double phi_c,
                   double dtf, double dtv, const double *mass_type, const int32_t *type,
                   double *phi)
{
    /* fix_aboundary_rho_meso.cu:88-94 (factors), :220-287 (kernel), in FP64 */
    double rc7 = pow(cut_phi, 7.0);
    double phi_factor = 105.0 / (16.0 * M_PI * rho_wall * rc7);
    double dw_factor = -315.0 / (4.0 * M_PI * rho_wall * rc7);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nlocal; ++i) {
        if (!(mask[i] & mobile_bit)) continue;
        double p = 0.0, nw[3] = {0, 0, 0};
        for (int k = 0; k < count[i]; ++k) {
            int j = table[(size_t)i * n_col + k];
            if (!(mask[j] & wall_bit)) continue;
            double d3[3] = {x[i] - xa[j], y[i] - ya[j], z[i] - za[j]};
            double rsq = d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2];
            if (!(rsq < cut_phi * cut_phi)) continue;
            double r = sqrt(rsq);
            if (r < 1e-10) r = 1e-10;
            double d = cut_phi - r;
            p += (cut_phi + 3.0 * r) * d * d * d * phi_factor;
            for (int a = 0; a < 3; ++a) nw[a] -= (r * d * d * dw_factor) * d3[a] / r;
        }
        phi[i] = p;
        if (p > phi_c) {
            double nn = sqrt(nw[0] * nw[0] + nw[1] * nw[1] + nw[2] * nw[2]);
            for (int a = 0; a < 3; ++a) nw[a] /= nn;
            double dtfm = dtf / mass_type[type[i] - 1];
            double v[3] = {vx[i], vy[i], vz[i]};
            double ox[3] = {x[i] - v[0] * dtfm, y[i] - v[1] * dtfm, z[i] - v[2] * dtfm};
            double t = v[0] * nw[0] + v[1] * nw[1] + v[2] * nw[2];
            if (t < 0) t = 0;
            vx[i] = -v[0] + 2 * t * nw[0];
            vy[i] = -v[1] + 2 * t * nw[1];
            vz[i] = -v[2] + 2 * t * nw[2];
            x[i] = ox[0] + dtv * vx[i];
            y[i] = ox[1] + dtv * vy[i];
            z[i] = ox[2] + dtv * vz[i];
        }
    }
}

void orc_force_mdpd(int nlocal, const float *pos4, const float *vel4, const double *rho,
                    const double *phi, const int32_t *mask, const int32_t *count,
                    const int32_t *table, int n_col, int ntype, const orc_mdpd_coeff *coeff,
                    double dt, int arb_bc, int mobile_bit, int wall_bit, double *f,
                    double *virial, double *epair)
{
    /* gpu_mdpd<evflag> (pair_mdpd_meso.cu:93-228) */
    const double dt_inv_sqrt = 1.0 / sqrt(dt);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nlocal; ++i) {
        double xi = pos4[4 * i], yi = pos4[4 * i + 1], zi = pos4[4 * i + 2];
        double vxi = vel4[4 * i], vyi = vel4[4 * i + 1], vzi = vel4[4 * i + 2];
        uint32_t si = f2u(vel4[4 * i + 3]);
        int ti = type_of(pos4, i);
        double fx = 0, fy = 0, fz = 0, vr[6] = {0, 0, 0, 0, 0, 0}, en = 0;
        for (int k = 0; k < count[i]; ++k) {
            int j = table[(size_t)i * n_col + k];
            /* r64 dx = coord1.x - coord2.x: an FP32 difference widened to FP64 */
            double dx = (float)(xi - pos4[4 * j]), dy = (float)(yi - pos4[4 * j + 1]),
                   dz = (float)(zi - pos4[4 * j + 2]);
            double rsq = dx * dx + dy * dy + dz * dz;
            const orc_mdpd_coeff *c = coeff + ti * ntype + type_of(pos4, j);
            if (!(rsq < c->cut * c->cut && rsq >= 1e-20)) continue;
            double r = sqrt(rsq);
            if (r < 1e-10) continue;
            double rinv = 1.0 / r;
            double dvx = (float)(vxi - vel4[4 * j]), dvy = (float)(vyi - vel4[4 * j + 1]),
                   dvz = (float)(vzi - vel4[4 * j + 2]);
            double dot = dx * dvx + dy * dvy + dz * dvz;
            double wc = 1.0 - r / c->cut;
            double wcr = 1.0 - r / c->cut_r;
            if (wcr < 0) wcr = 0;
            double rn = orc_gaussian_tea4(si, f2u(vel4[4 * j + 3]));
            double gam = c->gamma, sig = c->sigma;
            if (arb_bc && (mask[i] & mobile_bit) && (mask[j] & wall_bit)) {
                double p = phi[i] < 0.5 ? phi[i] : 0.5;
                double h = 1.0 - pow(2.088 * p * p * p + 1.478 * p, 0.25);
                if (h < 0.025) h = 0.025;
                h *= c->cut;
                double q = 1.0 - h / c->cut;
                double ratio = 1.0 + 0.187 * (c->cut / h - 1.0) - 0.093 * q * q * q;
                sig *= (double)sqrtf((float)ratio); /* sqrtf: FP32, as pair_mdpd_meso.cu:181 */
                gam *= ratio;
            }
            double fp = (c->A * wc + c->B * (rho[i] + rho[j]) * wcr) - gam * wc * wc * dot * rinv +
                        sig * wc * rn * dt_inv_sqrt;
            fp *= rinv;
            fx += dx * fp;
            fy += dy * fp;
            fz += dz * fp;
            if (virial || epair) {
                en += 0.5 * c->A * c->cut * wc * wc + 0.5 * c->B * c->cut_r * (rho[i] + rho[j]) * wcr * wcr;
                vr[0] += dx * dx * fp;
                vr[1] += dy * dy * fp;
                vr[2] += dz * dz * fp;
                vr[3] += dx * dy * fp;
                vr[4] += dx * dz * fp;
                vr[5] += dy * dz * fp;
            }
        }
        f[3 * i] = fx;
        f[3 * i + 1] = fy;
        f[3 * i + 2] = fz;
        if (virial)
            for (int a = 0; a < 6; ++a) virial[6 * i + a] = 0.5 * vr[a];
        if (epair) epair[i] = 0.5 * en;
    }
}

void orc_force_dpd(int nlocal, const float *pos4, const float *vel4, const int32_t *count,
                   const int32_t *table, int n_col, int ntype, const orc_dpd_coeff *coeff,
                   double dt, double *f, double *virial, double *epair)
{
    /* gpu_dpd<evflag> (pair_dpd_meso.cu:91-205), one partition */
    const double dt_inv_sqrt = 1.0 / sqrt(dt);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nlocal; ++i) {
        double xi = pos4[4 * i], yi = pos4[4 * i + 1], zi = pos4[4 * i + 2];
        double vxi = vel4[4 * i], vyi = vel4[4 * i + 1], vzi = vel4[4 * i + 2];
        uint32_t si = f2u(vel4[4 * i + 3]);
        int ti = type_of(pos4, i);
        double fx = 0, fy = 0, fz = 0, vr[6] = {0, 0, 0, 0, 0, 0}, en = 0;
        for (int k = 0; k < count[i]; ++k) {
            int j = table[(size_t)i * n_col + k];
            /* r64 dx = coord1.x - coord2.x: an FP32 difference widened to FP64 */
            double dx = (float)(xi - pos4[4 * j]), dy = (float)(yi - pos4[4 * j + 1]),
                   dz = (float)(zi - pos4[4 * j + 2]);
            double rsq = dx * dx + dy * dy + dz * dz;
            const orc_dpd_coeff *c = coeff + ti * ntype + type_of(pos4, j);
            if (!(rsq < c->cutsq && rsq >= 1e-20)) continue;
            double rn = orc_gaussian_tea4(si, f2u(vel4[4 * j + 3]));
            double r = sqrt(rsq);
            double rinv = 1.0 / r;
            double dvx = (float)(vxi - vel4[4 * j]), dvy = (float)(vyi - vel4[4 * j + 1]),
                   dvz = (float)(vzi - vel4[4 * j + 2]);
            double dot = dx * dvx + dy * dvy + dz * dvz;
            double wc = 1.0 - r * c->cutinv;
            double wr = c->expw == 1.0 ? wc : pow(wc, c->expw);
            double fp = c->a0 * wc - c->gamma * wr * wr * dot * rinv + c->sigma * wr * rn * dt_inv_sqrt;
            fp *= rinv;
            fx += dx * fp;
            fy += dy * fp;
            fz += dz * fp;
            if (virial || epair) {
                vr[0] += dx * dx * fp;
                vr[1] += dy * dy * fp;
                vr[2] += dz * dz * fp;
                vr[3] += dx * dy * fp;
                vr[4] += dx * dz * fp;
                vr[5] += dy * dz * fp;
                en += 0.5 * c->a0 * c->cut * wc * wc;
            }
        }
        f[3 * i] = fx;
        f[3 * i + 1] = fy;
        f[3 * i + 2] = fz;
        if (virial)
            for (int a = 0; a < 6; ++a) virial[6 * i + a] = 0.5 * vr[a];
        if (epair) epair[i] = 0.5 * en;
    }
}

/* ===================================================================== */
/* full single-box engine (CPU baseline)                                 */
/* ===================================================================== */

struct orc_sim {
    orc_sim_params p;
    orc_box box;
    int n, nghost, gcap;
    double *x, *y, *z, *vx, *vy, *vz, *f, *xh, *yh, *zh;
    int32_t *tag, *type, *mask;
    double *rho, *phi;        /* locals + ghosts */
    double *xa, *ya, *za;     /* absolute coords of locals + ghosts */
    int32_t *gsrc, *gimg, *gmask;
    float *pos4, *vel4;
    int32_t *count, *table;
    double *virial, *epair;
    int64_t step, nbuild;
    double cutforce;
};

static void sim_alloc_ghosts(orc_sim *s, int cap)
{
    free(s->gsrc);
    free(s->gimg);
    s->gcap = cap;
    s->gsrc = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap);
    s->gimg = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap);
    size_t na = (size_t)(s->n + cap);
    s->rho = (double *)realloc(s->rho, sizeof(double) * na);
    s->phi = (double *)realloc(s->phi, sizeof(double) * na);
    s->gmask = (int32_t *)realloc(s->gmask, sizeof(int32_t) * na);
    s->xa = (double *)realloc(s->xa, sizeof(double) * na);
    s->ya = (double *)realloc(s->ya, sizeof(double) * na);
    s->za = (double *)realloc(s->za, sizeof(double) * na);
    s->pos4 = (float *)realloc(s->pos4, sizeof(float) * 4 * na);
    s->vel4 = (float *)realloc(s->vel4, sizeof(float) * 4 * na);
}

orc_sim *orc_sim_create(const orc_sim_params *p, int n, const double *x, const double *v,
                        const int32_t *tag, const int32_t *type, const int32_t *mask)
{
    orc_sim *s = (orc_sim *)calloc(1, sizeof(orc_sim));
    s->p = *p;
    s->n = n;
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
    double cf = 0;
    for (int a = 0; a < p->ntype * p->ntype; ++a) {
        double c = p->style == 0 ? p->mcoeff[a].cut : p->dcoeff[a].cut;
        if (c > cf) cf = c;
    }
    s->cutforce = cf;
    orc_box_setup(&s->box, p->lo, p->hi, cf, p->skin, p->rho_est, n);
    size_t nn = (size_t)(n > 0 ? n : 1);
    double **arr[10] = {&s->x, &s->y, &s->z, &s->vx, &s->vy, &s->vz, &s->xh, &s->yh, &s->zh, &s->epair};
    for (int a = 0; a < 10; ++a) *arr[a] = (double *)calloc(nn, sizeof(double));
    s->f = (double *)calloc(3 * nn, sizeof(double));
    s->virial = (double *)calloc(6 * nn, sizeof(double));
    s->tag = (int32_t *)malloc(sizeof(int32_t) * nn);
    s->type = (int32_t *)malloc(sizeof(int32_t) * nn);
    s->mask = (int32_t *)malloc(sizeof(int32_t) * nn);
    s->count = (int32_t *)malloc(sizeof(int32_t) * nn);
    s->table = (int32_t *)malloc(sizeof(int32_t) * nn * (size_t)s->box.n_col);
    for (int i = 0; i < n; ++i) {
        s->x[i] = x[3 * i];
        s->y[i] = x[3 * i + 1];
        s->z[i] = x[3 * i + 2];
        s->vx[i] = v[3 * i];
        s->vy[i] = v[3 * i + 1];
        s->vz[i] = v[3 * i + 2];
        s->tag[i] = tag[i];
        s->type[i] = type[i];
        s->mask[i] = mask[i];
    }
    sim_alloc_ghosts(s, n / 2 + 1024);
    return s;
}

void orc_sim_destroy(orc_sim *s)
{
    if (!s) return;
    void *ptrs[] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->f, s->xh, s->yh, s->zh, s->tag,
                    s->type, s->mask, s->rho, s->phi, s->xa, s->ya, s->za, s->gsrc, s->gimg,
                    s->gmask, s->pos4, s->vel4, s->count, s->table, s->virial, s->epair};
    for (size_t a = 0; a < sizeof(ptrs) / sizeof(ptrs[0]); ++a) free(ptrs[a]);
    free(s);
}

static void permute_d(double *a, const int32_t *perm, int n, double *tmp)
{
    for (int i = 0; i < n; ++i) tmp[i] = a[perm[i]];
    memcpy(a, tmp, sizeof(double) * (size_t)n);
}

static void permute_i(int32_t *a, const int32_t *perm, int n, int32_t *tmp)
{
    for (int i = 0; i < n; ++i) tmp[i] = a[perm[i]];
    memcpy(a, tmp, sizeof(int32_t) * (size_t)n);
}

static int sim_rebuild(orc_sim *s)
{
    /* mvv_meso.cu:338-395: pbc, sort_local + permute, borders, neighbor build */
    int n = s->n;
    orc_pbc(&s->box, n, s->x, s->y, s->z);
    uint64_t *key = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n + 1));
    int32_t *perm = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    orc_reorder_keys(&s->box, n, s->x, s->y, s->z, key, NULL);
    orc_stable_sort_u64(n, key, perm);
    double *tmp = (double *)malloc(sizeof(double) * (size_t)(3 * n + 1));
    double *darr[] = {s->x, s->y, s->z, s->vx, s->vy, s->vz};
    for (int a = 0; a < 6; ++a) permute_d(darr[a], perm, n, tmp);
    for (int a = 0; a < 3; ++a) {
        for (int i = 0; i < n; ++i) tmp[i] = s->f[3 * perm[i] + a];
        for (int i = 0; i < n; ++i) s->f[3 * i + a] = tmp[i];
    }
    int32_t *itmp = (int32_t *)tmp;
    permute_i(s->tag, perm, n, itmp);
    permute_i(s->type, perm, n, itmp);
    permute_i(s->mask, perm, n, itmp);
    int nbulk = n;
    uint64_t bmask = 0;
    {
        int nbits;
        orc_reorder_keys(&s->box, 0, s->x, s->y, s->z, key, &nbits);
        bmask = 1ULL << (nbits - 1);
    }
    for (int i = 0; i < n; ++i)
        if (key[perm[i]] & bmask) {
            nbulk = i;
            break;
        }
    free(key);
    free(perm);
    free(tmp);
    int ng;
    while ((ng = orc_ghosts(&s->box, n, nbulk, s->x, s->y, s->z, s->gcap, s->gsrc, s->gimg)) < 0)
        sim_alloc_ghosts(s, s->gcap * 2);
    s->nghost = ng;
    for (int i = 0; i < n + ng; ++i) {
        double pxyz[3];
        int src = i < n ? i : s->gsrc[i - n];
        image_xyz(&s->box, s->x, s->y, s->z, src, i < n ? 13 : s->gimg[i - n], pxyz);
        s->xa[i] = pxyz[0];
        s->ya[i] = pxyz[1];
        s->za[i] = pxyz[2];
        s->gmask[i] = s->mask[src];
    }
    orc_pack_pos(&s->box, n, ng, s->x, s->y, s->z, s->type, s->gsrc, s->gimg, s->pos4);
    int ovf = orc_build_list(&s->box, n, n + ng, s->xa, s->ya, s->za, s->pos4, s->count, NULL,
                             s->table);
    for (int i = 0; i < n; ++i) {
        s->xh[i] = s->x[i];
        s->yh[i] = s->y[i];
        s->zh[i] = s->z[i];
    }
    s->nbuild++;
    return ovf ? 1 : 0;
}

static void sim_pack(orc_sim *s, uint32_t seed_now)
{
    int n = s->n, na = n + s->nghost;
    for (int i = 0; i < na; ++i) {
        int src = i < n ? i : s->gsrc[i - n];
        double pxyz[3];
        image_xyz(&s->box, s->x, s->y, s->z, src, i < n ? 13 : s->gimg[i - n], pxyz);
        s->xa[i] = pxyz[0];
        s->ya[i] = pxyz[1];
        s->za[i] = pxyz[2];
        s->pos4[4 * i] = (float)(pxyz[0] - s->box.cen[0]);
        s->pos4[4 * i + 1] = (float)(pxyz[1] - s->box.cen[1]);
        s->pos4[4 * i + 2] = (float)(pxyz[2] - s->box.cen[2]);
        s->pos4[4 * i + 3] = u2f((uint32_t)(s->type[src] - 1));
        s->vel4[4 * i] = (float)s->vx[src];
        s->vel4[4 * i + 1] = (float)s->vy[src];
        s->vel4[4 * i + 2] = (float)s->vz[src];
    }
    for (int i = 0; i < na; ++i) {
        int src = i < n ? i : s->gsrc[i - n];
        uint32_t sg;
        if (s->p.style == 0)
            sg = orc_premix_tea(orc_brev((uint32_t)s->tag[src]), seed_now, 32);
        else
            orc_sig_dpd(1, &s->tag[src], &s->vel4[4 * i], seed_now, &sg);
        s->vel4[4 * i + 3] = u2f(sg);
    }
}

static void sim_forces(orc_sim *s, int ev)
{
    int n = s->n;
    uint32_t sn = orc_seed_now(s->p.seed, s->step);
    double *mt = s->p.mass_type;
    if (s->p.style == 0) {
        sim_pack(s, 0);
        orc_density(n, s->pos4, s->count, s->table, s->box.n_col, s->mask, s->p.rho_groupbit,
                    s->p.cut_rho, mt, s->rho);
        for (int g = 0; g < s->nghost; ++g) s->rho[n + g] = s->rho[s->gsrc[g]];
        for (int g = 0; g < s->nghost; ++g) s->phi[n + g] = s->phi[s->gsrc[g]];
        sim_pack(s, sn);
        orc_force_mdpd(n, s->pos4, s->vel4, s->rho, s->phi, s->gmask, s->count, s->table,
                       s->box.n_col, s->p.ntype, s->p.mcoeff, s->p.dt, s->p.arb_bc,
                       s->p.mobile_bit, s->p.wall_bit, s->f, ev ? s->virial : NULL,
                       ev ? s->epair : NULL);
    } else {
        sim_pack(s, sn);
        orc_force_dpd(n, s->pos4, s->vel4, s->count, s->table, s->box.n_col, s->p.ntype,
                      s->p.dcoeff, s->p.dt, s->f, ev ? s->virial : NULL, ev ? s->epair : NULL);
    }
    /* addforce/meso (fix_addforce_meso.cu:72-90) */
    for (int i = 0; i < n; ++i)
        if (s->mask[i] & s->p.body_groupbit)
            for (int a = 0; a < 3; ++a) s->f[3 * i + a] += s->p.body_force[a];
}

int orc_sim_setup(orc_sim *s)
{
    for (int i = 0; i < s->n + s->gcap; ++i) s->phi[i] = 0.0;
    int e = sim_rebuild(s);
    sim_forces(s, 1);
    return e;
}

int orc_sim_run(orc_sim *s, int64_t nsteps)
{
    int n = s->n;
    const double dtf = 0.5 * s->p.dt, dtv = s->p.dt;
    const double trig = 0.25 * s->p.skin * s->p.skin; /* neighbor.cpp:237 */
    int err = 0;
    for (int64_t it = 0; it < nsteps; ++it) {
        s->step++;
        /* initial_integrate (fix_nve_meso.cu:62-95) */
        for (int i = 0; i < n; ++i) {
            if (!(s->mask[i] & s->p.nve_groupbit)) continue;
            double dtfm = dtf * orc_rcp(s->p.mass_type[s->type[i] - 1]);
            s->vx[i] = fma(dtfm, s->f[3 * i], s->vx[i]);
            s->vy[i] = fma(dtfm, s->f[3 * i + 1], s->vy[i]);
            s->vz[i] = fma(dtfm, s->f[3 * i + 2], s->vz[i]);
            s->x[i] = fma(dtv, s->vx[i], s->x[i]);
            s->y[i] = fma(dtv, s->vy[i], s->y[i]);
            s->z[i] = fma(dtv, s->vz[i], s->z[i]);
        }
        if (s->p.arb_bc) {
            orc_aboundary(n, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->xa, s->ya, s->za,
                          s->gmask, s->count, s->table, s->box.n_col, s->p.mobile_bit,
                          s->p.wall_bit, s->p.cut_phi, s->p.rho_wall, s->p.phi_c, dtf, dtv,
                          s->p.mass_type, s->type, s->phi);
        }
        /* rebuild trigger: exact max displacement (neighbor.cpp:1244-1322) */
        int flag = 0;
        for (int i = 0; i < n; ++i) {
            double dx = s->x[i] - s->xh[i], dy = s->y[i] - s->yh[i], dz = s->z[i] - s->zh[i];
            if (dx * dx + dy * dy + dz * dz > trig) {
                flag = 1;
                break;
            }
        }
        if (flag) err |= sim_rebuild(s);
        /* energy and virial on the run's last step, from that step's own force call (a LAMMPS
         * thermo step sets eflag/vflag on it; no extra force evaluation) */
        sim_forces(s, it == nsteps - 1);
        /* final_integrate (fix_nve_meso.cu:157-178) */
        for (int i = 0; i < n; ++i) {
            if (!(s->mask[i] & s->p.nve_groupbit)) continue;
            double dtfm = dtf * orc_rcp(s->p.mass_type[s->type[i] - 1]);
            s->vx[i] = fma(dtfm, s->f[3 * i], s->vx[i]);
            s->vy[i] = fma(dtfm, s->f[3 * i + 1], s->vy[i]);
            s->vz[i] = fma(dtfm, s->f[3 * i + 2], s->vz[i]);
        }
    }
    return err;
}

void orc_sim_get(const orc_sim *s, double *x, double *v, double *f, double *rho)
{
    for (int i = 0; i < s->n; ++i) {
        int t = s->tag[i] - 1;
        if (x) {
            x[3 * t] = s->x[i];
            x[3 * t + 1] = s->y[i];
            x[3 * t + 2] = s->z[i];
        }
        if (v) {
            v[3 * t] = s->vx[i];
            v[3 * t + 1] = s->vy[i];
            v[3 * t + 2] = s->vz[i];
        }
        if (f)
            for (int a = 0; a < 3; ++a) f[3 * t + a] = s->f[3 * i + a];
        if (rho) rho[t] = s->rho[i];
    }
}

int64_t orc_sim_step(const orc_sim *s) { return s->step; }
int64_t orc_sim_nbuild(const orc_sim *s) { return s->nbuild; }

void orc_sim_thermo(orc_sim *s, double out[14])
{
    /* T: sum m v^2 / (3 N kB) over the nve group (compute_temp_meso.cu:58-101),
     * virial trace, pair energy (from the last step's force call: setup and the last step of
     * every run compute them), total momentum, and the pressure tensor times the volume,
     * sum m v_a v_b + sum of the per-atom virials over all atoms (xx yy zz xy xz yz: the
     * library's thermo ptensor times V).  Nothing is recomputed: a force evaluation here
     * would replace the step's forces with ones from the full-step velocities and perturb the
     * next step */
    double ke = 0, vir = 0, pe = 0, px = 0, py = 0, pz = 0, pt[6] = {0, 0, 0, 0, 0, 0};
    int cnt = 0;
    for (int i = 0; i < s->n; ++i) {
        double m = s->p.mass_type[s->type[i] - 1];
        if (s->mask[i] & s->p.nve_groupbit) {
            ke += m * (s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
            cnt++;
        }
        vir += s->virial[6 * i] + s->virial[6 * i + 1] + s->virial[6 * i + 2];
        pe += s->epair[i];
        px += m * s->vx[i];
        py += m * s->vy[i];
        pz += m * s->vz[i];
        const double v[3] = {s->vx[i], s->vy[i], s->vz[i]};
        const int ab[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
        for (int q = 0; q < 6; ++q) pt[q] += m * v[ab[q][0]] * v[ab[q][1]] + s->virial[6 * i + q];
    }
    out[0] = cnt > 1 ? ke / (3.0 * cnt - 3.0) : 0.0; /* dof = 3N - 3 (extra_dof) */
    out[1] = vir;
    out[2] = pe;
    out[3] = px;
    out[4] = py;
    out[5] = pz;
    out[6] = (double)s->nbuild;
    out[7] = (double)s->step;
    for (int q = 0; q < 6; ++q) out[8 + q] = pt[q];
}

/* correctly rounded fused multiply-add, for checks written in Python */
double orc_fma(double a, double b, double c) { return fma(a, b, c); }
