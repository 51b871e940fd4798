/*
 * CPU oracle for the USER-MESO DPD/mDPD timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle that the CUDA path is
 * compared against, and the CPU baseline timed beside it.  Nothing in the
 * product (libmdpd.so) links, loads or calls it.
 *
 * Every function restates, in plain C with FP64 arithmetic (FP32 where the
 * reference decides set membership in FP32), the algorithm of the reference
 * file:line cited beside it.  Paths are relative to the reference project root.
 *
 * Pins (see tests/test_oracle_pins.py):
 *   - TEA words: against the reference's own math header compiled unmodified
 *     on the host (src/USER-MESO/math_meso.h:436-463), golden file
 *     tests/golden/tea_words.json.
 *   - gaussian_TEA<4> values: against the same header's device function run
 *     on a B200 (tests/golden/ref_device.json, key "gauss").
 *   - FP contraction of the binning, reorder-key and pair-distance expressions:
 *     against nvcc's own code for those expressions on a B200
 *     (tests/golden/ref_device.json, keys "dr2", "bin_expr", "sub_expr").
 *   - statistics: the static-contact-angle deck's density profiles
 *     (examples/v2.5/static_contact_angle_in_a_slit_nano_channel/out.profile.a_-*).
 */
#ifndef MDPD_ORACLE_H
#define MDPD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- counter-based RNG (math_meso.h:436-473) ---------------- */
uint32_t orc_brev(uint32_t x);
uint32_t orc_premix_tea(uint32_t v0, uint32_t v1, int rounds);
/* seed_now = premix_TEA<64>(seed, ntimestep)   (pair_mdpd_meso.cu:295-297) */
uint32_t orc_seed_now(uint32_t seed, int64_t ntimestep);
/* mDPD signature premix_TEA<32>(__brev(tag), seed_now) (atom_vec_mdpd_atomic_meso.cu:166) */
void orc_sig_mdpd(int n, const int32_t *tag, uint32_t seed_now, uint32_t *sig);
/* DPD signature seed ^ premix_TEA<16>(__brev(tag), mantissa(v))  (atom_vec_meso.cu:164) */
void orc_sig_dpd(int n, const int32_t *tag, const float *vel4, uint32_t seed_now, uint32_t *sig);
/* gaussian_TEA<4>(si > sj, si, sj), FP64, bit-exact restatement (math_meso.h:465-473) */
double orc_gaussian_tea4(uint32_t si, uint32_t sj);
void orc_gaussian_batch(int n, const uint32_t *si, const uint32_t *sj, double *out);
/* the reference's own reciprocal (math_meso.h:229-237) */
double orc_rcp(double x);
uint64_t orc_morton3(uint32_t x, uint32_t y, uint32_t z);

/* ---------------- box / bins (neighbor_meso.cu:771-853, neigh_list_meso.cu:78-90) ------- */
typedef struct orc_box {
    double lo[3], hi[3], prd[3], cen[3];
    double skin, cutneighmax, cutghost;
    double binsize[3], bininv[3];
    int mbin[3];
    int n_col;                 /* list row padding, ceil32(expected_neigh_count) */
    float rc2_core, rc2_tail;  /* (float)pow(cutneighmax-skin,2), (float)pow(cutneighmax,2) */
    double expected_neigh_count;
} orc_box;

/* rho_est > 0: atom_style mdpd/atomic/meso density estimate; else nlocal/volume */
void orc_box_setup(orc_box *b, const double lo[3], const double hi[3], double cutforce,
                   double skin, double rho_est, int nlocal);

/* Domain::pbc wrap of local positions into [lo,hi) */
void orc_pbc(const orc_box *b, int n, double *x, double *y, double *z);

/* number of slabs (of 6) containing each particle (comm_meso.cu:195-261, comm.cpp:585-610) */
void orc_borderness(const orc_box *b, int n, const double *x, const double *y, const double *z,
                    int *border);
/* 2-level reorder key, gpu_build_reorder_keypair<1> (atom_meso.cu:271-311,346-387) */
void orc_reorder_keys(const orc_box *b, int n, const double *x, const double *y, const double *z,
                      uint64_t *key, int *nbits);
/* stable ascending sort of keys: perm[k] = original index of k-th element */
void orc_stable_sort_u64(int n, const uint64_t *key, int32_t *perm);

/* ghost images, MesoComm::borders swap order (comm_meso.cu:42-193).
 * Locals must already be ordered bulk-then-border (n_bulk = first border index).
 * For each ghost g: src[g] = local index, img[g] = (sx+1) + 3*(sy+1) + 9*(sz+1).
 * Ghost coordinate = x[src] + sx*prd[0] (FP64), as pack_border_vel does.
 * Returns the ghost count, or -1 if cap is exceeded. */
int orc_ghosts(const orc_box *b, int nlocal, int n_bulk, const double *x, const double *y,
               const double *z, int cap, int32_t *src, int32_t *img);

/* FP32 pack relative to the box centre: pos4 = ((float)(x-c), ..., int_as_float(type-1))
 * for locals then ghosts (gpu_merge_xvt_mdpd, atom_vec_mdpd_atomic_meso.cu:140-175) */
void orc_pack_pos(const orc_box *b, int nlocal, int nghost, const double *x, const double *y,
                  const double *z, const int32_t *type, const int32_t *src, const int32_t *img,
                  float *pos4);

/* bin id of every local+ghost (gpu_assign_bin_id, neighbor_meso.cu:390-425) */
void orc_bin_ids(const orc_box *b, int nlocal, int nall, const double *x, const double *y,
                 const double *z, uint32_t *bin);

/* full neighbor list (gpu_build_neighbor_list + join, neigh_build_meso.cu:17-127,188-232):
 * row-major table[i*n_col + k]; core (dr2 <= rc2_core) entries in stencil order first, then
 * skin entries in reverse stencil order.  Returns 0, or the first overflowing local + 1. */
void orc_reduce_rows(int nlocal, int ncol, const int32_t *count, const int32_t *table,
                     const float *pos4, const int32_t *gimg, float rn2, int32_t *out_count,
                     int32_t *out_table);
void orc_aboundary_meso(int nlocal, const float *pos4, const int32_t *mask_all, const int32_t *count,
                        const int32_t *table, int ncol, int mobile_bit, int wall_bit, double rho0, double sigma,
                        double dt, double *vx, double *vy, double *vz, double *fx, double *fy, double *fz);
int orc_build_list(const orc_box *b, int nlocal, int nall, const double *x, const double *y,
                   const double *z, const float *pos4, int32_t *count, int32_t *count_core,
                   int32_t *table);

/* the FP32 squared distance exactly as nvcc contracts dx*dx+dy*dy+dz*dz */
float orc_dr2f(float dx, float dy, float dz);
double orc_fma(double a, double b, double c);

/* ---------------- pair passes (row-major list, any order) ---------------- */
typedef struct orc_mdpd_coeff {   /* per type pair (pair_mdpd_meso.h:15-23) */
    double cut, cut_r, A, B, gamma, sigma;
} orc_mdpd_coeff;

typedef struct orc_dpd_coeff {    /* per type pair (pair_dpd_meso.h:15-23) */
    double cut, cutsq, cutinv, expw, a0, gamma, sigma;
} orc_dpd_coeff;

/* local density (gpu_compute_rho, fix_aboundary_rho_meso.cu:119-165), FP64 */
void orc_density(int nlocal, const float *pos4, const int32_t *count, const int32_t *table,
                 int n_col, const int32_t *mask, int groupbit, double cut_rho,
                 const double *mass_type, double *rho);

/* wall volume fraction and bounce-back (gpu_aboundary, fix_aboundary_rho_meso.cu:220-287).
 * xa: absolute coordinates (FP64) of locals+ghosts; updates x, v (locals) and phi. */
void orc_aboundary(int nlocal, double *x, double *y, double *z, double *vx, double *vy,
                   double *vz, const double *xa, const double *ya, const double *za,
                   const int32_t *mask, const int32_t *count, const int32_t *table, int n_col,
                   int mobile_bit, int wall_bit, double cut_phi, double rho_wall, double phi_c,
                   double dtf, double dtv, const double *mass_type, const int32_t *type,
                   double *phi);

/* mDPD force (gpu_mdpd<evflag>, pair_mdpd_meso.cu:93-228), FP64 on FP32 packed inputs.
 * rho/phi/mask are indexed over locals+ghosts.  f: 3*nlocal, virial: 6*nlocal or NULL,
 * epair: nlocal or NULL.  Forces are written (not accumulated). */
void orc_force_mdpd(int nlocal, const float *pos4, const float *vel4, const double *rho,
                    const double *phi, const int32_t *mask, const int32_t *count,
                    const int32_t *table, int n_col, int ntype, const orc_mdpd_coeff *coeff,
                    double dt, int arb_bc, int mobile_bit, int wall_bit, double *f,
                    double *virial, double *epair);

/* classic DPD force (gpu_dpd<evflag>, pair_dpd_meso.cu:91-205) */
void orc_force_dpd(int nlocal, const float *pos4, const float *vel4, const int32_t *count,
                   const int32_t *table, int n_col, int ntype, const orc_dpd_coeff *coeff,
                   double dt, double *f, double *virial, double *epair);

/* ---------------- full single-box engine (the CPU baseline) ---------------- */
typedef struct orc_sim orc_sim;

typedef struct orc_sim_params {
    int style;               /* 0 = mdpd, 1 = dpd */
    int ntype;
    double lo[3], hi[3];
    double skin, dt, kT;
    uint32_t seed;
    double rho_est;
    double cut_rho;          /* mdpd density cut (fix aboundary/rho/meso cut_rho) */
    double mass_type[8];
    orc_mdpd_coeff mcoeff[64];   /* ntype*ntype, row-major */
    orc_dpd_coeff dcoeff[64];
    int nve_groupbit;        /* mask bit of the nve/meso group */
    int rho_groupbit;        /* mask bit of the density fix group */
    double body_force[3];    /* addforce/meso */
    int body_groupbit;
    int arb_bc, mobile_bit, wall_bit;
    double cut_phi, rho_wall, phi_c;
    int nthreads;            /* OpenMP threads, 0 = default */
} orc_sim_params;

orc_sim *orc_sim_create(const orc_sim_params *p, int n, const double *x, const double *v,
                        const int32_t *tag, const int32_t *type, const int32_t *mask);
void orc_sim_destroy(orc_sim *s);
/* LAMMPS run setup: rebuild + density + force (ModifiedVerlet::setup, mvv_meso.cu:203-283) */
int orc_sim_setup(orc_sim *s);
/* n velocity-Verlet steps (ModifiedVerlet::run, mvv_meso.cu:309-572). Returns 0 or error. */
int orc_sim_run(orc_sim *s, int64_t nsteps);
/* state in tag order */
void orc_sim_get(const orc_sim *s, double *x, double *v, double *f, double *rho);
int64_t orc_sim_step(const orc_sim *s);
int64_t orc_sim_nbuild(const orc_sim *s);
/* thermo: temperature (compute_temp_meso.cu:58-101), virial trace sum, PE, momentum, build
 * count, step, and the pressure tensor times the volume (xx yy zz xy xz yz) */
void orc_sim_thermo(orc_sim *s, double out[14]);

#ifdef __cplusplus
}
#endif
#endif
