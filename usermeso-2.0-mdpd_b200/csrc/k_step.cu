// Per-step kernels: fused velocity-Verlet integrate + FP32 pack + ghost refresh,
// the mDPD density pass, the mDPD/DPD force pass (with the final half-kick fused into
// its epilogue) and the deterministic FP64 thermo reductions.
//
// Reference semantics:
//   integrate      fix_nve_meso.cu:62-95 and :157-178 (FP64 x,v; dtfm = dtf*rcp(m))
//   pack           atom_vec_mdpd_atomic_meso.cu:140-175, atom_vec_meso.cu:142-168
//   ghosts         periodic images x + s*prd of comm_meso.cu:42-193, built on the device
//   wall           fix_aboundary_rho_meso.cu:220-287
//   density        fix_aboundary_rho_meso.cu:119-165
//   force (mdpd)   pair_mdpd_meso.cu:93-228
//   force (dpd)    pair_dpd_meso.cu:91-205
//   rebuild check  neighbor.cpp:1216-1231 (decide), :1244-1322 (check_distance)
#include "engine.h"
#include "kernels.h"
#include "pair.cuh"

#include <cstdio>

namespace mdpd {

__device__ __forceinline__ bool last_block(int *done)
{
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    return s_last;
}

// ---------------------------------------------------------------------------
// integrate: initial half-kick + drift (+ wall bounce-back), displacement check,
// FP32 pack of locals and their ghost images.  The last block decides the rebuild
// per box (LAMMPS Neighbor::decide) and sets the graph's conditional.
// ---------------------------------------------------------------------------
// resident blocks per SM of the integrate pass (the wall variant holds the wall normal sums)
constexpr int integrate_blocks(bool wall) { return wall ? 5 : 8; }

// packed position and velocity of ghost g, image `code` of a local at (x, y, z)
__device__ __forceinline__ void put_ghost(const BoxDesc &B, int g, int code, double x, double y, double z,
                                          float w, float4 vv)
{
    B.pos[B.nlocal + g] = make_float4((float)(x + (code % 3 - 1) * B.prd[0] - B.cen[0]),
                                      (float)(y + ((code / 3) % 3 - 1) * B.prd[1] - B.cen[1]),
                                      (float)(z + (code / 9 - 1) * B.prd[2] - B.cen[2]), ghost_w(w, code));
    B.vel[B.nlocal + g] = vv;
}

template <bool WALL, int STYLE>
__global__ void __launch_bounds__(kUnit, integrate_blocks(WALL)) k_integrate(BoxDesc *__restrict__ boxes,
                                                     const Unit *__restrict__ units, int nunits,
                                                     int nbox, int *done,
                                                     cudaGraphConditionalHandle cond, int use_cond)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        const int c = B.st->cur;
        const int i = U.begin + threadIdx.x;
        bool moved = false;
        if (i < U.end) {
            // every load of the particle is issued before the first store (the compiler may not
            // move a load above a store to a possibly aliased array): one memory round trip
            const BoxState &S = *B.st;
            const long long step = S.step + 1;
            const int n_bulk = S.n_bulk;
            const bool sn_cached = S.sn_ok && S.sn_step == step && S.sn_seed == B.seed;
            const uint32_t sn_c = S.sn;
            const int t = B.type[c][i], m = B.mask[c][i], tag = B.tag[c][i];
            double x = B.x[c][0][i], y = B.x[c][1][i], z = B.x[c][2][i];
            double vx = B.v[c][0][i], vy = B.v[c][1][i], vz = B.v[c][2][i];
            const float4 f = B.f[c][i];
            const double hx = B.xh[0][i], hy = B.xh[1][i], hz = B.xh[2][i];
            const bool edge = i >= n_bulk;
            const int g0 = edge ? B.gfirst[i] : 0;
            const int g1 = edge ? min(B.gfirst[i + 1], B.ghost_cap) : 0;  // an overflowed build is reported, never written past
            int code8[8];  // image codes of the first ghosts (7 at most unless a side is < 2 cutoffs)
#pragma unroll
            for (int q = 0; q < 8; ++q) code8[q] = g0 + q < g1 ? B.gimg[g0 + q] : 13;
            const double dtfm = B.dtfm[t - 1];
            if (m & B.nve_bit) {
                // the body force in FP64 (added to FP32 forces it would round the same way for
                // every particle of a binade: a bias)
                const bool body = m & B.body_bit;
                vx = __fma_rn(dtfm, (double)f.x + (body ? B.body[0] : 0.0), vx);
                vy = __fma_rn(dtfm, (double)f.y + (body ? B.body[1] : 0.0), vy);
                vz = __fma_rn(dtfm, (double)f.z + (body ? B.body[2] : 0.0), vz);
                x = __fma_rn(B.dtv, vx, x);
                y = __fma_rn(B.dtv, vy, y);
                z = __fma_rn(B.dtv, vz, z);
            }
            if (WALL && B.wall_fix && (m & B.mobile_bit)) {
                // wall volume fraction and normal from frozen wall neighbours (old list)
                const float cx = (float)x, cy = (float)y, cz = (float)z;
                double phi_i = 0.0;
                float nx = 0.f, ny = 0.f, nz = 0.f;
                const int n = MDPD_IDX(B.count[i], B.n_col + 1);
                const float cp = B.cut_phi;
                for (int k = 0; k < n; ++k) {
                    const int j = MDPD_IDX(B.table[list_addr(i, k, B.n_col)] & kEntryIndexMask, n_all(B));
                    const float4 pj = B.pos[j];
                    if (!(pflags(pj) & 2)) continue;
                    int s = j, code = 13;
                    if (j >= B.nlocal) {
                        s = MDPD_IDX(B.gsrc[j - B.nlocal], B.nlocal);
                        code = B.gimg[j - B.nlocal];
                    }
                    const float jx = (float)(B.x[c][0][s] + (code % 3 - 1) * B.prd[0]);
                    const float jy = (float)(B.x[c][1][s] + ((code / 3) % 3 - 1) * B.prd[1]);
                    const float jz = (float)(B.x[c][2][s] + (code / 9 - 1) * B.prd[2]);
                    const float dx = cx - jx, dy = cy - jy, dz = cz - jz;
                    const float rsq = dist2(dx, dy, dz);
                    if (rsq < cp * cp) {
                        const float rinv = rsqrtf(rsq);
                        const float r = fmaxf(rsq * rinv, 1e-10f);
                        const float d = cp - r;
                        phi_i += (double)((cp + 3.f * r) * d * d * d * B.phi_factor);
                        const float w = r * d * d * B.dw_factor * rinv;
                        nx -= w * dx;
                        ny -= w * dy;
                        nz -= w * dz;
                    }
                }
                B.phi[c][i] = (float)phi_i;
                if (phi_i > B.phi_c) {
                    const float nn = rsqrtf(nx * nx + ny * ny + nz * nz);
                    nx *= nn, ny *= nn, nz *= nn;
                    const double dtfm = B.dtf / B.mass[t - 1];
                    const double ox = x - vx * dtfm, oy = y - vy * dtfm, oz = z - vz * dtfm;
                    const double tt = fmax(0.0, vx * nx + vy * ny + vz * nz);
                    vx = -vx + 2.0 * tt * nx;
                    vy = -vy + 2.0 * tt * ny;
                    vz = -vz + 2.0 * tt * nz;
                    x = ox + B.dtv * vx;
                    y = oy + B.dtv * vy;
                    z = oz + B.dtv * vz;
                }
            }
            B.v[c][0][i] = vx, B.v[c][1][i] = vy, B.v[c][2][i] = vz;
            B.x[c][0][i] = x, B.x[c][1][i] = y, B.x[c][2][i] = z;
            const double ddx = x - hx, ddy = y - hy, ddz = z - hz;
            moved = ddx * ddx + ddy * ddy + ddz * ddz > B.triggersq;
            // pack
            const uint32_t sn = sn_cached ? sn_c : seed_now(B.seed, step);  // box-uniform branch
            const float w = pack_w(B, t, m);
            const float4 p = make_float4((float)(x - B.cen[0]), (float)(y - B.cen[1]),
                                         (float)(z - B.cen[2]), w);
            const float fvx = (float)vx, fvy = (float)vy, fvz = (float)vz;
            const uint32_t sg = STYLE == 0 ? sig_mdpd(tag, sn) : sig_dpd(tag, fvx, fvy, fvz, sn);
            const float4 vv = make_float4(fvx, fvy, fvz, __uint_as_float(sg));
            B.pos[i] = p;
            B.vel[i] = vv;
            if (edge) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (g0 + q < g1) put_ghost(B, g0 + q, code8[q], x, y, z, w, vv);
                for (int g = g0 + 8; g < g1; ++g) put_ghost(B, g, B.gimg[g], x, y, z, w, vv);
            }
        }
        if (__syncthreads_or(moved) && threadIdx.x == 0) atomicOr(&B.st->moved, 1);
    }
    if (last_block(done)) {
        int any = 0;
        for (int b = threadIdx.x; b < nbox; b += blockDim.x) {
            BoxState *S = boxes[b].st;
            const BoxDesc &B = boxes[b];
            const int moved = atomicExch(&S->moved, 0);
            const int ago = S->ago + 1;
            int rb = 0;
            if (ago >= B.delay && ago % B.every == 0) rb = B.check ? moved : 1;
            S->rebuild = rb;
            S->ago = rb ? 0 : ago;
            // this step's seed (for a rebuild's pack) and the next step's, once per box instead
            // of once per particle (64 TEA rounds)
            const long long s1 = S->step + 1;
            const uint32_t used =
                S->sn_ok && S->sn_step == s1 && S->sn_seed == B.seed ? S->sn : seed_now(B.seed, s1);
            S->step = s1;
            S->sn_prev = used;
            S->sn = seed_now(B.seed, s1 + 1);
            S->sn_step = s1 + 1;
            S->sn_seed = B.seed;
            S->sn_ok = 1;
            any |= rb;
        }
        any = __syncthreads_or(any);
        if (threadIdx.x == 0) {
            *done = 0;
            if (any) done[3] += 1;  // steps that ran the rebuild body
            if (use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
        }
    }
}

void launch_integrate(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c,
                      int *done, cudaGraphConditionalHandle cond, int use_cond)
{
    const int full = c.sms * integrate_blocks(c.wall);  // one resident wave, grid-stride over units
    int grid = u.local.n < full ? u.local.n : full;
    if (grid < 1) grid = 1;
    if (c.wall) {
        if (c.style == 0)
            k_integrate<true, 0><<<grid, kUnit, 0, s>>>(boxes, u.local.d, u.local.n, u.nbox, done, cond, use_cond);
        else
            k_integrate<true, 1><<<grid, kUnit, 0, s>>>(boxes, u.local.d, u.local.n, u.nbox, done, cond, use_cond);
    } else {
        if (c.style == 0)
            k_integrate<false, 0><<<grid, kUnit, 0, s>>>(boxes, u.local.d, u.local.n, u.nbox, done, cond, use_cond);
        else
            k_integrate<false, 1><<<grid, kUnit, 0, s>>>(boxes, u.local.d, u.local.n, u.nbox, done, cond, use_cond);
    }
}

__global__ void k_force_rebuild_flag(BoxDesc *boxes, int nbox, int value)
{
    for (int b = threadIdx.x; b < nbox; b += blockDim.x) {
        boxes[b].st->rebuild = value;
        if (value) boxes[b].st->ago = 0;
    }
}

void launch_force_rebuild_flag(cudaStream_t s, BoxDesc *boxes, int nbox, int value)
{
    k_force_rebuild_flag<<<1, 256, 0, s>>>(boxes, nbox, value);
}

// ---------------------------------------------------------------------------
// fix aboundary/meso (fix_aboundary_meso.cu:186-281, gpu_aboundary_v2 at end_of_step): for a
// particle of the fix's group, project it half a kick and one drift ahead, sum a Gaussian
// density of the wall particles among its whole list row, and where that density passes rho0/2
// remove the parts of v and f pointing into the wall.  The reference passes the row length as
// dev_pair_count_core, which its list build's join (gpu_join_neigh_list,
// neigh_build_meso.cu:188-204) has set to the core plus skin count: every entry of the row.
// FP32 as the reference, with its contractions spelled out.
// ---------------------------------------------------------------------------
// a.x*b.x + a.y*b.y + a.z*b.z as nvcc contracts it (the form of dist2)
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz)
{
    return __fmaf_rn(az, bz, __fmaf_rn(ax, bx, __fmul_rn(ay, by)));
}

__global__ void __launch_bounds__(kUnit) k_aboundary_meso(BoxDesc *__restrict__ boxes,
                                                          const Unit *__restrict__ units, int nunits)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!B.ab_mobile_bit) continue;
        const int i = U.begin + threadIdx.x;
        if (i >= U.end) continue;
        const int c = B.st->cur;
        const int m = B.mask[c][i];
        if (!(m & B.ab_mobile_bit)) continue;
        const float dt = (float)B.dtv;
        const float hs = (float)(0.5 * (double)dt);
        const bool body = m & B.body_bit;
        const float4 fp = B.f[c][i];
        // the total force (pair + fix addforce/meso), as the reference's f holds it
        const double fx = (double)fp.x + (body ? B.body[0] : 0.0), fy = (double)fp.y + (body ? B.body[1] : 0.0),
                     fz = (double)fp.z + (body ? B.body[2] : 0.0);
        const double vx = B.v[c][0][i], vy = B.v[c][1][i], vz = B.v[c][2][i];
        const float3 v0 = make_float3((float)vx, (float)vy, (float)vz);
        const float3 f0 = make_float3((float)fx, (float)fy, (float)fz);
        const float4 x0 = B.pos[i];
        const float3 vp = make_float3(__fmaf_rn(hs, f0.x, v0.x), __fmaf_rn(hs, f0.y, v0.y), __fmaf_rn(hs, f0.z, v0.z));
        const float3 c1 = make_float3(__fmaf_rn(dt, vp.x, x0.x), __fmaf_rn(dt, vp.y, x0.y), __fmaf_rn(dt, vp.z, x0.z));
        const float sig = B.ab_sigma, nf = B.ab_nfactor;
        const float ex = __fdiv_rn(-0.5f, sig);
        float rho_w = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
        const int n = MDPD_IDX(B.count[i], B.n_col + 1);
        for (int k = 0; k < n; ++k) {
            const int j = MDPD_IDX(B.table[list_addr(i, k, B.n_col)] & kEntryIndexMask, n_all(B));
            const int mj = j < B.nlocal ? B.mask[c][j] : B.mask[c][MDPD_IDX(B.gsrc[j - B.nlocal], B.nlocal)];
            if (!(mj & B.ab_wall_bit)) continue;
            const float4 c2 = B.pos[j];
            const float dx = c1.x - c2.x, dy = c1.y - c2.y, dz = c1.z - c2.z;
            const float rsq = dist2(dx, dy, dz);
            const float w = __fmul_rn(nf, expf(__fmul_rn(ex, rsq)));
            rho_w += w;
            const float ws = __fdiv_rn(w, sig);
            gx = __fmaf_rn(dx, ws, gx);
            gy = __fmaf_rn(dy, ws, gy);
            gz = __fmaf_rn(dz, ws, gz);
        }
        if (rho_w > 0.5f * B.ab_rho0) {
            const float inv = rsqrtf(dot3(gx, gy, gz, gx, gy, gz));
            const float ex_ = -(gx * inv), ey_ = -(gy * inv), ez_ = -(gz * inv);  // e = -normalize(grad)
            const float vd = fmaxf(0.f, dot3(v0.x, v0.y, v0.z, ex_, ey_, ez_));
            const float fd = fmaxf(0.f, dot3(f0.x, f0.y, f0.z, ex_, ey_, ez_));
            B.v[c][0][i] = vx - (double)(2.f * vd * ex_);
            B.v[c][1][i] = vy - (double)(2.f * vd * ey_);
            B.v[c][2][i] = vz - (double)(2.f * vd * ez_);
            // f keeps the pair force; the body force is added again by the kicks
            B.f[c][i] = make_float4((float)(fx - (double)(2.f * fd * ex_) - (body ? B.body[0] : 0.0)),
                                    (float)(fy - (double)(2.f * fd * ey_) - (body ? B.body[1] : 0.0)),
                                    (float)(fz - (double)(2.f * fd * ez_) - (body ? B.body[2] : 0.0)), fp.w);
        }
    }
}

void launch_aboundary_meso(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u)
{
    if (u.local.n <= 0) return;
    k_aboundary_meso<<<u.local.n, kUnit, 0, s>>>(boxes, u.local.d, u.local.n);
}

// ---------------------------------------------------------------------------
// density pass: rho_i = m_i * 15/(2 pi h^5) * sum_{r<h} (h - r)^2 over the list.
// TPP threads per particle split the list and combine with shuffles.
// ---------------------------------------------------------------------------
template <int TPP>
__global__ void __launch_bounds__(kUnit *TPP, 16 / TPP) k_density(const BoxDesc *__restrict__ boxes,
                                                         const Unit *__restrict__ units, int nunits)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        const int i = U.begin + threadIdx.x / TPP;
        const int t = threadIdx.x % TPP;
        float acc = 0.f;
        const bool live = i < U.end;
        const int c = B.st->cur;
        const bool in_group = live && (B.mask[c][i] & B.rho_bit);
        if (in_group) {
            const float4 pi = B.pos[i];
            const float h = B.cut_rho, h2 = h * h;
            const int n = MDPD_IDX(B.count[i], B.n_col + 1);
            const int ncol = B.n_col;
            const int *row = B.table + ((unsigned)(i & ~31) * (unsigned)ncol + (unsigned)(i & 31));
            // four independent index -> position gather chains in flight per thread
            for (int k0 = t; k0 < n; k0 += 4 * TPP) {
                int j[4];
                float4 pj[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int k = k0 + q * TPP;
                    j[q] = k < n ? MDPD_IDX(__ldcs(row + 32 * k) & kEntryIndexMask, n_all(B)) : -1;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) pj[q] = j[q] >= 0 ? __ldg(&B.pos[j[q]]) : make_float4(1e30f, 0, 0, 0);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    // branchless: (h - r)^2 for 1e-20 <= r^2 < h^2, else 0
                    const float dx = pi.x - pj[q].x, dy = pi.y - pj[q].y, dz = pi.z - pj[q].z;
                    const float rsq = dist2(dx, dy, dz);
                    const float d = (rsq < h2 && rsq >= 1e-20f) ? h - rsq * rsqrtf(rsq) : 0.f;
                    acc = __fmaf_rn(d, d, acc);
                }
            }
        }
#pragma unroll
        for (int o = TPP / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (in_group && t == 0) {
            const float r = (float)(B.mass[ptype(B.pos[i])] * B.rho_factor) * acc;
            B.rho[i] = r;
            if (i >= B.st->n_bulk) {
                const int g1 = min(B.gfirst[i + 1], B.ghost_cap);
                for (int g = B.gfirst[i]; g < g1; ++g) B.rho[B.nlocal + g] = r;
            }
        }
    }
}

void launch_density(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c)
{
    const int grid = u.local.n < c.sms * 16 ? (u.local.n > 0 ? u.local.n : 1) : c.sms * 16;
    if (c.half) {
        launch_density_half(s, boxes, u, c);
        return;
    }
    switch (c.tpp_density) {
    case 2: k_density<2><<<grid, kUnit * 2, 0, s>>>(boxes, u.local.d, u.local.n); break;
    case 4: k_density<4><<<grid, kUnit * 4, 0, s>>>(boxes, u.local.d, u.local.n); break;
    default: k_density<1><<<grid, kUnit, 0, s>>>(boxes, u.local.d, u.local.n); break;
    }
}

// ---------------------------------------------------------------------------
// force pass.  Per list entry: FP32 distance test against the type-pair cutoff; inside
// it, the conservative + dissipative + random force with the pairwise gaussian of the
// two signatures.  Epilogue (t==0): store f, final half-kick (FP64 v, body force in FP64).
// ---------------------------------------------------------------------------
constexpr int kQueue = 16;  // list entries tested per phase-1 round of the force pass

// 8 blocks of 128 threads per SM (64 registers): measured faster on a wall-coupled box than 10
// blocks at 48 registers, which spilled
template <int TPP, int STYLE, bool EXACT, bool EV, bool WALLC, bool UNI>
__global__ void __launch_bounds__(kUnit *TPP, 8 / TPP) k_force(const BoxDesc *__restrict__ boxes,
                                                       const Unit *__restrict__ units, int nunits, int kick)
{
    __shared__ PairCoeff s_coeff[kMaxTypes * kMaxTypes];
    __shared__ double s_red[kUnit * TPP / 32][7];
    __shared__ int s_q[kQueue][kUnit * TPP];  // per-thread queue of in-range neighbours
    int cur_box = -1;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (U.box != cur_box) {
            __syncthreads();
            const int nc = B.ntype * B.ntype;
            for (int q = threadIdx.x; q < nc; q += blockDim.x) s_coeff[q] = B.coeff[q];
            cur_box = U.box;
            __syncthreads();
        }
        const int ntype = B.ntype;
        const int i = U.begin + threadIdx.x / TPP;
        const int t = threadIdx.x % TPP;
        const bool live = i < U.end;
        float fx = 0.f, fy = 0.f, fz = 0.f;
        EvAcc ev = {0, 0, 0, 0, 0, 0, 0};
        float4 pi = make_float4(0, 0, 0, 0);
        const int c = B.st->cur;
        if (live) {
            pi = B.pos[i];
            const float4 vi = B.vel[i];
            const uint32_t si = __float_as_uint(vi.w);
            const int ti = ptype(pi);
            const float rho_i = STYLE == 0 ? B.rho[i] : 0.f;
            float wall_ratio = 1.f, wall_sqrt = 1.f;
            const bool i_mobile = WALLC && (pflags(pi) & 1);
            if (WALLC && i_mobile) {
                // gamma/sigma scaling of (mobile, wall) pairs from phi_i (pair_mdpd_meso.cu:171-185);
                // with h = h'*rcw the ratio depends on h' only
                const float ph = fminf(B.phi[c][i], 0.5f);
                const float hp = fmaxf(1.f - sqrtf(sqrtf(2.088f * ph * ph * ph + 1.478f * ph)), 0.025f);
                const float q = 1.f - hp;
                wall_ratio = 1.f + 0.187f * (1.f / hp - 1.f) - 0.093f * q * q * q;
                wall_sqrt = sqrtf(wall_ratio);
            }
            const float dtis = B.dt_inv_sqrt;
            const int n = MDPD_IDX(B.count[i], B.n_col + 1);
            const int ncol = B.n_col;
            const int *row = B.table + ((unsigned)(i & ~31) * (unsigned)ncol + (unsigned)(i & 31));
            for (int kb = t; kb < n; kb += kQueue * TPP) {
                // phase 1: distance test of up to kQueue entries, four gathers in flight;
                // in-range neighbours are queued (this thread's column of s_q)
                int nq = 0;
#pragma unroll
                for (int b4 = 0; b4 < kQueue; b4 += 4) {
                    int j[4];
                    float4 pj[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int k = kb + (b4 + q) * TPP;
                        j[q] = k < n ? MDPD_IDX(__ldcs(row + 32 * k) & kEntryIndexMask, n_all(B)) : -1;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        pj[q] = j[q] >= 0 ? __ldg(&B.pos[j[q]]) : make_float4(1e30f, 0, 0, 0);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float dx = pi.x - pj[q].x, dy = pi.y - pj[q].y, dz = pi.z - pj[q].z;
                        const float rsq = dist2(dx, dy, dz);
                        const int cid = UNI ? 0 : ti * ntype + ptype(pj[q]);
                        if (j[q] >= 0 && rsq < s_coeff[cid].cutsq && rsq >= 1e-20f)
                            s_q[nq++][threadIdx.x] = j[q];
                    }
                }
                // phase 2: forces of the queued neighbours, in list order
                for (int q = 0; q < nq; ++q) {
                    const int j = s_q[q][threadIdx.x];
                    const float4 pj = __ldg(&B.pos[j]);
                    pair_term<STYLE, EXACT, EV, WALLC>(B, s_coeff[UNI ? 0 : ti * ntype + ptype(pj)], j, pj, pi, vi, si,
                                                       rho_i, i_mobile, wall_ratio, wall_sqrt, dtis, fx, fy, fz, ev);
                }
            }
        }
#pragma unroll
        for (int o = TPP / 2; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(0xffffffffu, fx, o);
            fy += __shfl_xor_sync(0xffffffffu, fy, o);
            fz += __shfl_xor_sync(0xffffffffu, fz, o);
            if (EV) {
                ev.vxx += __shfl_xor_sync(0xffffffffu, ev.vxx, o);
                ev.vyy += __shfl_xor_sync(0xffffffffu, ev.vyy, o);
                ev.vzz += __shfl_xor_sync(0xffffffffu, ev.vzz, o);
                ev.vxy += __shfl_xor_sync(0xffffffffu, ev.vxy, o);
                ev.vxz += __shfl_xor_sync(0xffffffffu, ev.vxz, o);
                ev.vyz += __shfl_xor_sync(0xffffffffu, ev.vyz, o);
                ev.pe += __shfl_xor_sync(0xffffffffu, ev.pe, o);
            }
        }
        if (live && t == 0) {
            const int m = B.mask[c][i];
            if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&B.st->status, kErrNonFinite);
            B.f[c][i] = make_float4(fx, fy, fz, 0.f);  // the pair force; the body force is in the kicks
            if (kick && (m & B.nve_bit)) {
                const double dtfm = B.dtfm[ptype(pi)];
                const bool body = m & B.body_bit;
                B.v[c][0][i] = __fma_rn(dtfm, (double)fx + (body ? B.body[0] : 0.0), B.v[c][0][i]);
                B.v[c][1][i] = __fma_rn(dtfm, (double)fy + (body ? B.body[1] : 0.0), B.v[c][1][i]);
                B.v[c][2][i] = __fma_rn(dtfm, (double)fz + (body ? B.body[2] : 0.0), B.v[c][2][i]);
            }
        }
        if (EV) {
            // per-unit FP64 partials in a fixed order (deterministic)
            double vals[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (live && t == 0) {
                vals[0] = 0.5 * ev.vxx, vals[1] = 0.5 * ev.vyy, vals[2] = 0.5 * ev.vzz;
                vals[3] = 0.5 * ev.vxy, vals[4] = 0.5 * ev.vxz, vals[5] = 0.5 * ev.vyz;
                vals[6] = 0.5 * ev.pe;
            }
            const double tot = warp_sum_spread(vals);  // the warp's total of value lane / 4
            const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
            if ((lane & 3) == 0 && (lane >> 2) < 7) s_red[w][lane >> 2] = tot;
            __syncthreads();
            if (threadIdx.x < 7) {
                double a = 0.0;
                for (int ww = 0; ww < (int)(blockDim.x / 32); ++ww) a += s_red[ww][threadIdx.x];
                B.partial[(size_t)(U.begin / kUnit) * kPartialStride + 1 + threadIdx.x] = a;
            }
            __syncthreads();
        }
    }
}

template <int TPP, int STYLE, bool EXACT, bool EV>
static void force_launch_wall(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, int grid, int wallc, int kick,
                              int uniform)
{
    if (wallc)
        k_force<TPP, STYLE, EXACT, EV, true, false><<<grid, kUnit * TPP, 0, s>>>(boxes, u.local.d, u.local.n, kick);
    else if (uniform)
        k_force<TPP, STYLE, EXACT, EV, false, true><<<grid, kUnit * TPP, 0, s>>>(boxes, u.local.d, u.local.n, kick);
    else
        k_force<TPP, STYLE, EXACT, EV, false, false><<<grid, kUnit * TPP, 0, s>>>(boxes, u.local.d, u.local.n, kick);
}

template <int TPP, int STYLE>
static void force_launch_tpp(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, int grid,
                             const StepConfig &c, int ev, int kick)
{
    if (c.exact_rng) {
        if (ev) force_launch_wall<TPP, STYLE, true, true>(s, boxes, u, grid, c.wall_coupling, kick, c.uniform_types);
        else force_launch_wall<TPP, STYLE, true, false>(s, boxes, u, grid, c.wall_coupling, kick, c.uniform_types);
    } else {
        if (ev) force_launch_wall<TPP, STYLE, false, true>(s, boxes, u, grid, c.wall_coupling, kick, c.uniform_types);
        else force_launch_wall<TPP, STYLE, false, false>(s, boxes, u, grid, c.wall_coupling, kick, c.uniform_types);
    }
}

template <int STYLE>
static void force_launch_style(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, int grid,
                               const StepConfig &c, int ev, int kick)
{
    switch (c.tpp_force) {
    case 2: force_launch_tpp<2, STYLE>(s, boxes, u, grid, c, ev, kick); break;
    case 4: force_launch_tpp<4, STYLE>(s, boxes, u, grid, c, ev, kick); break;
    default: force_launch_tpp<1, STYLE>(s, boxes, u, grid, c, ev, kick); break;
    }
}

void launch_force(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int ev, int kick)
{
    if (c.half) {
        launch_force_half(s, boxes, u, c, ev, kick);
        return;
    }
    const int grid = u.local.n < c.sms * 16 ? (u.local.n > 0 ? u.local.n : 1) : c.sms * 16;
    if (c.style == 0) force_launch_style<0>(s, boxes, u, grid, c, ev, kick);
    else force_launch_style<1>(s, boxes, u, grid, c, ev, kick);
}

// ---------------------------------------------------------------------------
// thermo: per-unit kinetic energy / momentum partials, then per-box sums in unit order.
// slots: 0 sum m v^2 (all), 1..6 virial xx yy zz xy xz yz (force pass), 7 pair energy,
// 8..10 momentum, 11 sum m v^2 over the nve group, 12..17 kinetic tensor xx yy zz xy xz yz.
// ---------------------------------------------------------------------------
// A block takes a group of kThermoGroup consecutive units of a box (the group's first unit; the
// others of the group are skipped): each thread sums its particles i, i + kUnit, ... in that
// order, then the warp and block trees; the sums go to the group's first partial row and zeros
// to the others, so the per-box tree of k_thermo_sum is unchanged.  The structure depends only
// on particle indices: the sums are the same bits for any grid.
constexpr int kThermoGroup = 8;
__global__ void __launch_bounds__(kUnit) k_thermo_units(const BoxDesc *__restrict__ boxes,
                                                        const Unit *__restrict__ units, int nunits)
{
    constexpr int NQ = 11;  // sums, padded to 16 for the warp reduction
    __shared__ double s_red[kUnit / 32][NQ];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const int row = U.begin / kUnit;
        if (row % kThermoGroup != 0) continue;  // taken by its group's first unit
        const BoxDesc &B = boxes[U.box];
        const int c = B.st->cur;
        const int end = min(U.begin + kThermoGroup * kUnit, B.nlocal);
        double vals[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) vals[q] = 0.0;
#pragma unroll 4
        for (int i = U.begin + threadIdx.x; i < end; i += kUnit) {
            const int t = B.type[c][i];
            const double m = B.mass[t - 1];
            const double vx = B.v[c][0][i], vy = B.v[c][1][i], vz = B.v[c][2][i];
            const double ke = m * (vx * vx + vy * vy + vz * vz);
            vals[0] += ke;
            vals[1] += m * vx, vals[2] += m * vy, vals[3] += m * vz;
            if (B.mask[c][i] & B.nve_bit) vals[4] += ke;
            vals[5] += m * vx * vx, vals[6] += m * vy * vy, vals[7] += m * vz * vz;
            vals[8] += m * vx * vy, vals[9] += m * vx * vz, vals[10] += m * vy * vz;
        }
        const double tot = warp_sum_spread(vals);  // the warp's total of value lane / 2
        const int lane = threadIdx.x & 31;
        if ((lane & 1) == 0 && (lane >> 1) < NQ) s_red[threadIdx.x / 32][lane >> 1] = tot;
        __syncthreads();
        const int rows = (B.nlocal + kUnit - 1) / kUnit;
        for (int k = threadIdx.x; k < NQ * kThermoGroup; k += blockDim.x) {
            const int q = k % NQ, r = row + k / NQ;
            if (r >= rows) continue;
            double a = 0.0;
            if (r == row)
                for (int w = 0; w < kUnit / 32; ++w) a += s_red[w][q];
            B.partial[(size_t)r * kPartialStride + (q == 0 ? 0 : q + 7)] = a;  // slots 0, 8..17
        }
        __syncthreads();
    }
}

__global__ void k_thermo_sum(const BoxDesc *__restrict__ boxes, int nbox, double *out)
{
    // one block per box: fixed-order tree over the unit partials
    __shared__ double s[256];
    const int b = blockIdx.x;
    if (b >= nbox) return;
    const BoxDesc &B = boxes[b];
    const int nunit = (B.nlocal + kUnit - 1) / kUnit;
    for (int q = 0; q < kPartialStride; ++q) {
        double a = 0.0;
        for (int k = threadIdx.x; k < nunit; k += blockDim.x) a += B.partial[(size_t)k * kPartialStride + q];
        s[threadIdx.x] = a;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[(size_t)b * kPartialStride + q] = s[0];
        __syncthreads();
    }
}

__global__ void k_load_state(const double *__restrict__ xa, const double *__restrict__ va, int n, double *x0,
                             double *x1, double *x2, double *h0, double *h1, double *h2, double *v0, double *v1,
                             double *v2, int *tag, int *type, int *mask)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double a = xa[3 * i], b = xa[3 * i + 1], c = xa[3 * i + 2];
    x0[i] = h0[i] = a, x1[i] = h1[i] = b, x2[i] = h2[i] = c;
    v0[i] = va ? va[3 * i] : 0.0, v1[i] = va ? va[3 * i + 1] : 0.0, v2[i] = va ? va[3 * i + 2] : 0.0;
    if (tag) tag[i] = i + 1;
    if (type) type[i] = 1;
    if (mask) mask[i] = 1;
}

// splitmix64's output function (Steele, Lea and Flood, 2014): a counter-based hash
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// uniform in (0, 1) from draw k of the stream seed
__device__ __forceinline__ double unit_open(unsigned long long seed, unsigned long long k)
{
    return ((double)(mix64(seed ^ mix64(k)) >> 11) + 0.5) * 0x1p-53;
}

// particle i: draws 16 i .. 16 i + 8 (x, y, z, then a Box-Muller pair per velocity component);
// the velocity sum in 2^-32 fixed point (integer adds: the same total in any order)
__global__ void k_fill(Fill f, double3 blo, double3 bhi, int n, double *__restrict__ xa, double *__restrict__ va,
                       unsigned long long *mom)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    long long q[3] = {0, 0, 0};
    if (i < n) {
        const double lo[3] = {blo.x, blo.y, blo.z}, hi[3] = {bhi.x, bhi.y, bhi.z};
        const unsigned long long k0 = 16ull * (unsigned long long)i;
        for (int d = 0; d < 3; ++d) {
            double x = f.lo[d] + unit_open(f.seed, k0 + d) * (f.hi[d] - f.lo[d]);
            if (x >= hi[d]) x = lo[d];
            xa[3 * (size_t)i + d] = x;
            const double u1 = unit_open(f.seed, k0 + 3 + 2 * d), u2 = unit_open(f.seed, k0 + 4 + 2 * d);
            const double v = f.vscale * sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
            va[3 * (size_t)i + d] = v;
            q[d] = __double2ll_rn(v * 4294967296.0);
        }
    }
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) q[d] += __shfl_xor_sync(0xffffffffu, q[d], o);
        if ((threadIdx.x & 31) == 0) atomicAdd(mom + d, (unsigned long long)q[d]);
    }
}

__global__ void k_fill_center(int n, double *__restrict__ va, const unsigned long long *mom)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < 3; ++d) va[3 * (size_t)i + d] -= (double)(long long)mom[d] * 0x1p-32 / n;
}

void launch_fill(cudaStream_t s, const Fill &f, const double box_lo[3], const double box_hi[3], int n, double *xa,
                 double *va, unsigned long long *mom)
{
    if (n <= 0) return;
    const int g = (n + 255) / 256;
    k_fill<<<g, 256, 0, s>>>(f, make_double3(box_lo[0], box_lo[1], box_lo[2]),
                             make_double3(box_hi[0], box_hi[1], box_hi[2]), n, xa, va, mom);
    k_fill_center<<<g, 256, 0, s>>>(n, va, mom);
}

void launch_load_state(cudaStream_t s, const double *xa, const double *va, int n, double *const x[3],
                       double *const xh[3], double *const v[3], int *tag, int *type, int *mask)
{
    if (n > 0)
        k_load_state<<<(n + 255) / 256, 256, 0, s>>>(xa, va, n, x[0], x[1], x[2], xh[0], xh[1], xh[2], v[0], v[1],
                                                      v[2], tag, type, mask);
}

__global__ void k_gather_states(const BoxDesc *__restrict__ boxes, int nbox, BoxState *__restrict__ out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nbox) out[b] = *boxes[b].st;
}

void launch_gather_states(cudaStream_t s, const BoxDesc *boxes, int nbox, BoxState *out)
{
    if (nbox > 0) k_gather_states<<<(nbox + 127) / 128, 128, 0, s>>>(boxes, nbox, out);
}

__global__ void k_gather_by_tag(StateBuffers b, const BoxState *__restrict__ st, int n, double *__restrict__ xo,
                                double *__restrict__ vo)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = st->cur & 1;
    const int r = b.tag[c][i] - 1;
    if (r < 0 || r >= n) return;  // tags are 1..n by construction
    xo[3 * r] = b.x[c][0][i], xo[3 * r + 1] = b.x[c][1][i], xo[3 * r + 2] = b.x[c][2][i];
    vo[3 * r] = b.v[c][0][i], vo[3 * r + 1] = b.v[c][1][i], vo[3 * r + 2] = b.v[c][2][i];
}

void launch_gather_by_tag(cudaStream_t s, const StateBuffers &b, const BoxState *st, int n, double *xo, double *vo)
{
    if (n > 0) k_gather_by_tag<<<(n + 255) / 256, 256, 0, s>>>(b, st, n, xo, vo);
}

void launch_thermo(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, double *out, int *)
{
    const int grid = u.local.n < 148 * 8 ? (u.local.n > 0 ? u.local.n : 1) : 148 * 8;
    k_thermo_units<<<grid, kUnit, 0, s>>>(boxes, u.local.d, u.local.n);
    k_thermo_sum<<<u.nbox, 256, 0, s>>>(boxes, u.nbox, out);
}

// ---------------------------------------------------------------------------
// density profile (fix density/meso, fix_density_profile_meso.cpp:118-151)
// ---------------------------------------------------------------------------
__global__ void k_density_profile(const BoxDesc *__restrict__ boxes, const Unit *__restrict__ units,
                                  int nunits, int dim, int groupbit, double lo, double inv, int nbin,
                                  unsigned long long *counts)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        const int c = B.st->cur;
        const int i = U.begin + threadIdx.x;
        if (i < U.end && (B.mask[c][i] & groupbit)) {
            const int b = (int)floor((B.x[c][dim][i] - lo) * inv);
            if (b >= 0 && b < nbin) atomicAdd(&counts[b], 1ull);
        }
    }
}

void launch_density_profile(cudaStream_t s, const BoxDesc *boxes, int, const Unit *units, int nunits,
                            int dim, int groupbit, double lo, double inv, int nbin,
                            unsigned long long *counts)
{
    const int grid = nunits < 148 * 8 ? (nunits > 0 ? nunits : 1) : 148 * 8;
    k_density_profile<<<grid, kUnit, 0, s>>>(boxes, units, nunits, dim, groupbit, lo, inv, nbin, counts);
}

// ---------------------------------------------------------------------------
// pair RNG on explicit signature pairs (test hook)
// ---------------------------------------------------------------------------
__global__ void k_gaussian(const uint32_t *si, const uint32_t *sj, double *exact, float *fast, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (exact) exact[i] = gaussian_exact(si[i], sj[i]);
        if (fast) fast[i] = gaussian_fast(si[i], sj[i]);
    }
}

void launch_gaussian(cudaStream_t s, const uint32_t *si, const uint32_t *sj, double *exact, float *fast, int n)
{
    const int grid = (n + 255) / 256 < 148 * 8 ? ((n + 255) / 256 > 0 ? (n + 255) / 256 : 1) : 148 * 8;
    k_gaussian<<<grid, 256, 0, s>>>(si, sj, exact, fast, n);
}

}  // namespace mdpd
