// Per-pair force terms shared by the pair-pass kernels.
#pragma once

#include "mdpd_dev.cuh"

namespace mdpd {

struct EvAcc {
    float vxx, vyy, vzz, vxy, vxz, vyz, pe;
};

// one pair's contribution to particle i from the pair geometry and both particles' state
// (pair_mdpd_meso.cu:139-225, pair_dpd_meso.cu:126-187); the caller has checked
// cf.cutsq > rsq >= 1e-20
template <int STYLE, bool EXACT, bool EV, bool WALLC>
__device__ __forceinline__ void pair_core(const PairCoeff &cf, float dx, float dy, float dz, float rsq,
                                          const float4 &vi, const float4 &vj, uint32_t si, float rho_i,
                                          float rho_j, bool wall_scaled, float wall_ratio, float wall_sqrt,
                                          float dtis, float &fx, float &fy, float &fz, EvAcc &ev)
{
    // the hardware's approximate 1/sqrt refined by one Newton-Raphson step,
    // y1 = y0 + y0 (1 - x y0^2) / 2: the pair terms then carry ~1 ulp of FP32 error instead of the
    // approximation's few, which is what keeps a particle's summed force within 1e-5 of the FP64
    // reference where its pair forces nearly cancel
    const float y0 = rsqrtf(rsq);
    const float e = __fmaf_rn(-rsq * y0, y0, 1.f);
    const float rinv = __fmaf_rn(0.5f * e, y0, y0);
    const float r = rsq * rinv;
    if (r < 1e-10f) return;
    const float dvx = vi.x - vj.x, dvy = vi.y - vj.y, dvz = vi.z - vj.z;
    const float dot = __fmaf_rn(dz, dvz, __fmaf_rn(dy, dvy, dx * dvx));
    const float wc = 1.f - r * cf.inv_cut;
    float gam = cf.gamma, sig = cf.sigma;
    float rn;
    if (EXACT)
        rn = (float)gaussian_exact(si, __float_as_uint(vj.w));
    else
        rn = gaussian_fast(si, __float_as_uint(vj.w));
    float fpair;
    if (STYLE == 0) {
        const float wcr = fmaxf(1.f - r * cf.inv_cut_r, 0.f);
        if (WALLC && wall_scaled) {
            sig *= wall_sqrt;
            gam *= wall_ratio;
        }
        fpair = (cf.A * wc + cf.B * (rho_i + rho_j) * wcr) - gam * wc * wc * dot * rinv + sig * wc * rn * dtis;
        if (EV) ev.pe += cf.e_cut * wc * wc + cf.e_cut_r * (rho_i + rho_j) * wcr * wcr;
    } else {
        const float wr = cf.expw == 1.f ? wc : __powf(wc, cf.expw);
        fpair = cf.A * wc - gam * wr * wr * dot * rinv + sig * wr * rn * dtis;
        if (EV) ev.pe += cf.e_cut * wc * wc;
    }
    fpair *= rinv;
    fx = __fmaf_rn(dx, fpair, fx);
    fy = __fmaf_rn(dy, fpair, fy);
    fz = __fmaf_rn(dz, fpair, fz);
    if (EV) {
        ev.vxx += dx * dx * fpair;
        ev.vyy += dy * dy * fpair;
        ev.vzz += dz * dz * fpair;
        ev.vxy += dx * dy * fpair;
        ev.vxz += dx * dz * fpair;
        ev.vyz += dy * dz * fpair;
    }
}

// one pair's contribution to particle i, loading j's velocity and density only when the pair
// is inside the type-pair cutoff
template <int STYLE, bool EXACT, bool EV, bool WALLC>
__device__ __forceinline__ void pair_term(const BoxDesc &B, const PairCoeff &cf, int j, const float4 &pj,
                                          const float4 &pi, const float4 &vi, uint32_t si, float rho_i,
                                          bool i_mobile, float wall_ratio, float wall_sqrt, float dtis, float &fx,
                                          float &fy, float &fz, EvAcc &ev)
{
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    const float rsq = dist2(dx, dy, dz);
    if (!(rsq < cf.cutsq && rsq >= 1e-20f)) return;
    const float4 vj = __ldg(&B.vel[j]);
    const float rho_j = STYLE == 0 ? __ldg(&B.rho[j]) : 0.f;
    pair_core<STYLE, EXACT, EV, WALLC>(cf, dx, dy, dz, rsq, vi, vj, si, rho_i, rho_j,
                                       WALLC && i_mobile && (pflags(pj) & 2), wall_ratio, wall_sqrt, dtis, fx, fy,
                                       fz, ev);
}

}  // namespace mdpd
