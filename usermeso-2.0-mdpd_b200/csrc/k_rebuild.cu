// Neighbour rebuild pipeline, run for the boxes whose rebuild flag is set:
//
//   key      wrap into the box (MesoDomain::pbc, domain_meso.cu:58-110); 2-level reorder
//            key = border | Morton(bin) | Morton(16^3 sub-bin) (atom_meso.cu:271-311,346-387)
//            split into a bucket class (border, Morton rank of the bin) and a 12-bit sub key
//   sort     deterministic bucket sort: count -> scan -> scatter -> per-bucket sort by
//            (sub key, original index).  Equals the reference's stable LSD radix sort of the
//            full key (sort_meso.h:364-443), i.e. the same permutation.
//   permute  gather every per-particle array into the other buffer, pack FP32 state,
//            count ghost images of border particles, bin the locals
//   ghosts   periodic images x + s*prd of every particle within cutghost of a face
//            (MesoComm::borders, comm_meso.cu:42-193), binned with gpu_assign_bin_id's rule
//            (neighbor_meso.cu:390-425)
//   bins     locals+ghosts by bin, index order inside a bin: a local's place follows from its
//            reorder-class run; ghost images take atomic slots and bins holding them are sorted
//   list     warp per bin: 27-bin stencil candidates filtered against the box of up to 32
//            centres, then tested against each centre; every hit is written from the test
//            ballot (atomic-free) straight into the locally transposed table, reduced rows on
//            pair-once boxes (gpu_build_neighbor_list, neigh_build_meso.cu:17-127; layout
//            neigh_list_meso.cu:143-147)
#include <algorithm>
#include <mutex>

#include "kernels.h"

namespace mdpd {

enum { kSelCls = 0, kSelGhost = 1, kSelBin = 2 };

__device__ __forceinline__ bool rebuilding(const BoxDesc &B) { return B.st->rebuild != 0; }

// counter[idx] += 1 for each calling lane, one atomic per distinct idx among the converged lanes
// (particles of one bin or class mostly sit next to each other, so a warp's lanes share few
// counters); returns what a per-lane atomicAdd would have returned, in lane order within each idx
__device__ __forceinline__ int warp_add1(int *counter, int idx)
{
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, idx);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter + idx, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// ---------------------------------------------------------------------------
// R1: wrap + reorder key
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUnit) k_rb_key(const BoxDesc *__restrict__ boxes,
                                                  const Unit *__restrict__ units, int nunits)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int i = U.begin + threadIdx.x;
        if (i >= U.end) continue;
        const int c = B.st->cur;
        uint32_t bid[3], sub[3];
        bool border = false;
        double xs[3];  // all three loads before the first store (no round trip per axis)
        for (int d = 0; d < 3; ++d) xs[d] = B.x[c][d][i];
        for (int d = 0; d < 3; ++d) {
            double x = xs[d];
            if (x < B.lo[d]) x += B.prd[d];
            if (x >= B.hi[d]) {
                x -= B.prd[d];
                x = fmax(x, B.lo[d]);
            }
            if (!(x >= B.lo[d] && x < B.hi[d])) atomicOr(&B.st->status, kErrLost);
            B.x[c][d][i] = x;
            bid[d] = (uint32_t)clamp_bin(bin_coord(x, B.lo[d], B.bininv[d]), B.mbin[d]);
            const double off = __fma_rn(-(double)(uint32_t)(bid[d] - 1u), B.binsize[d], x);
            sub[d] = (uint32_t)clamp_bin((int)__dmul_rn(off, B.coord_inv[d]), 16);
            border |= (x <= B.lo[d] + B.cutghost) || (x >= B.hi[d] - B.cutghost);
        }
        const int bin = (int)(bid[0] + B.mbin[0] * (bid[1] + bid[2] * B.mbin[1]));
        const int cls = MDPD_IDX((border ? B.nbin : 0) + B.bin_rank[MDPD_IDX(bin, B.nbin)], 2 * B.nbin);
        B.cls_of[i] = cls;
        B.sub_of[i] = (int)morton3(sub[0], sub[1], sub[2]);
        warp_add1(B.cls_count, cls);
    }
}

// ---------------------------------------------------------------------------
// scans: per-box exclusive scans of a count array, three kernels without inter-block waits
// ---------------------------------------------------------------------------
template <int SEL> __device__ __forceinline__ int *scan_in(const BoxDesc &B)
{
    return SEL == kSelCls ? B.cls_count : SEL == kSelGhost ? B.gfirst : B.bin_count;
}
template <int SEL> __device__ __forceinline__ int scan_len(const BoxDesc &B)
{
    return SEL == kSelCls ? 2 * B.nbin : SEL == kSelGhost ? B.nlocal + 1 : B.nbin;
}

template <int SEL>
__global__ void __launch_bounds__(256) k_scan_reduce(const BoxDesc *__restrict__ boxes,
                                                     const Unit *__restrict__ units, int nunits)
{
    __shared__ int s_w[8];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int *in = scan_in<SEL>(B);
        int a = 0;
        for (int k = U.begin + threadIdx.x; k < U.end; k += 256) a += in[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x / 32] = a;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < 8; ++w) t += s_w[w];
            B.scan_part[U.begin / kScanChunk] = t;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int block_exclusive_scan_256(int v, int *s_w, int &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x / 32;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        int t = threadIdx.x < 8 ? s_w[threadIdx.x] : 0;
        for (int o = 1; o < 8; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (threadIdx.x < 8) s_w[8 + threadIdx.x] = t;
    }
    __syncthreads();
    total = s_w[15];
    const int base = w > 0 ? s_w[8 + w - 1] : 0;
    const int r = base + x - v;
    __syncthreads();
    return r;
}

template <int SEL>
__global__ void __launch_bounds__(256) k_scan_top(const BoxDesc *__restrict__ boxes, int nbox)
{
    __shared__ int s_w[16];
    const int b = blockIdx.x;
    if (b >= nbox) return;
    const BoxDesc &B = boxes[b];
    if (!rebuilding(B)) return;
    const int nch = (scan_len<SEL>(B) + kScanChunk - 1) / kScanChunk;
    int carry = 0;
    for (int base = 0; base < nch; base += 256) {
        const int k = base + threadIdx.x;
        const int v = k < nch ? B.scan_part[k] : 0;
        int total;
        const int ex = block_exclusive_scan_256(v, s_w, total);
        if (k < nch) B.scan_part[k] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) B.scan_part[nch] = carry;
}

template <int SEL>
__global__ void __launch_bounds__(256) k_scan_down(const BoxDesc *__restrict__ boxes,
                                                   const Unit *__restrict__ units, int nunits)
{
    __shared__ int s_w[16];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        int *in = scan_in<SEL>(B);
        const int n = scan_len<SEL>(B);
        int carry = B.scan_part[U.begin / kScanChunk];
        // 8 items per thread, blocked
        int v[8];
        const int k0 = U.begin + threadIdx.x * 8;
        int local = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            v[q] = (k0 + q < U.end) ? in[k0 + q] : 0;
            local += v[q];
        }
        int total;
        int ex = block_exclusive_scan_256(local, s_w, total) + carry;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = k0 + q;
            if (k < U.end) {
                if (SEL == kSelCls) {
                    B.cls_start[k] = ex;
                    B.cls_cursor[k] = ex;
                } else if (SEL == kSelGhost) {
                    in[k] = ex;
                } else {
                    B.bin_start[k] = ex;
                    B.bin_cursor[k] = ex;
                }
            }
            ex += v[q];
        }
        if (U.end == n && threadIdx.x == 255) {
            // totals: ghost count / bin_start[nbin] / class sentinel
            const int tot = ex;
            if (SEL == kSelGhost) B.st->nghost = tot;
            if (SEL == kSelBin) B.bin_start[n] = tot;
            if (SEL == kSelCls) B.cls_start[n] = tot;
        }
    }
}

// resident blocks per SM of the scan passes, from the occupancy API (init_rebuild_shapes)
static int g_scan_reduce[3] = {4, 4, 4}, g_scan_down[3] = {4, 4, 4};

template <int SEL>
static void scan(cudaStream_t s, BoxDesc *boxes, const UnitList &ul, int nbox, int sms)
{
    auto g = [&](int per_sm) { return ul.n < sms * per_sm ? (ul.n > 0 ? ul.n : 1) : sms * per_sm; };
    k_scan_reduce<SEL><<<g(g_scan_reduce[SEL]), 256, 0, s>>>(boxes, ul.d, ul.n);
    k_scan_top<SEL><<<nbox, 256, 0, s>>>(boxes, nbox);
    k_scan_down<SEL><<<g(g_scan_down[SEL]), 256, 0, s>>>(boxes, ul.d, ul.n);
}

// ---------------------------------------------------------------------------
// R3: scatter locals into their reorder buckets
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUnit) k_rb_scatter_cls(const BoxDesc *__restrict__ boxes,
                                                          const Unit *__restrict__ units, int nunits)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int i = U.begin + threadIdx.x;
        if (i >= U.end) continue;
        const int p = warp_add1(B.cls_cursor, MDPD_IDX(B.cls_of[i], 2 * B.nbin));
        B.perm[MDPD_IDX(p, B.nlocal)] = i;
    }
}

// ---------------------------------------------------------------------------
// R4 / R10: warp per bucket, order members by (sub key, index) or by index
// ---------------------------------------------------------------------------
// Position of particle i as the list build reads it from bpos: x, y, z and, in .w, its list word:
// i for a local or an upper ghost image, ~i for a lower ghost image.  As a signed integer the word
// orders a candidate against a centre (a local) as pair-once ownership does: a candidate whose
// word is above the centre's index is owned by the centre (a local above it, or an upper image;
// a lower image is negative, below every centre), and only the centre itself has an equal word.
__device__ __forceinline__ float4 list_pos(const float4 &p, int i, int nlocal)
{
    const int wd = i < nlocal || (pflags(p) & kUpperImage) ? i : ~i;
    return make_float4(p.x, p.y, p.z, __int_as_float(wd));
}

// One bucket's members in (key, index) order by the whole warp: the ranks from a shared-memory
// copy of the keys (buckets of up to kClassMax members).
template <int MODE>
__device__ __forceinline__ void bucket_warp(const BoxDesc &B, int *arr, int s, int n, int lane,
                                            unsigned long long *key)
{
    const int lim = MODE == 0 ? B.nlocal : n_all(B);
    for (int e = lane; e < n; e += 32) {
        const int idx = MDPD_IDX(arr[s + e], lim);
        key[e] = MODE == 0 ? (((unsigned long long)(uint32_t)B.sub_of[idx] << 32) | (uint32_t)idx)
                           : (unsigned long long)(uint32_t)idx;
    }
    __syncwarp();
    for (int e = lane; e < n; e += 32) {
        const unsigned long long k = key[e];
        int rank = 0;
        for (int q = 0; q < n; ++q) rank += key[q] < k;
        const int idx = (int)(uint32_t)k;
        arr[s + rank] = idx;
        if (MODE == 1) B.bpos[s + rank] = list_pos(B.pos[idx], idx, B.nlocal);
    }
    __syncwarp();
}

// Buckets are taken four at a time per warp, one per group of 8 lanes holding up to 4 members
// each: a bucket of up to 32 members (the usual case: a reorder class is one bin's interior or
// border locals, ~14 at rho 6.05) is ordered with shuffles inside its group, so the warp waits
// once for the loads of four buckets; a larger one is ordered by the whole warp afterwards.
constexpr int kGroupSlots = 4;  // members per lane of an 8-lane group
template <int MODE>  // 0: reorder classes -> perm, 1: bins -> bin_order + bpos
__global__ void __launch_bounds__(256, 4) k_rb_bucket(const BoxDesc *__restrict__ boxes,
                                                   const Unit *__restrict__ units, int nunits)
{
    __shared__ unsigned long long s_key[8][kClassMax];
    const int lane = threadIdx.x & 31, w = threadIdx.x / 32;
    const int grp = lane >> 3, l8 = lane & 7;
    unsigned long long *key = s_key[w];
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        int *cnt = MODE == 0 ? B.cls_count : B.bin_count;
        const int *start = MODE == 0 ? B.cls_start : B.bin_start;
        int *arr = MODE == 0 ? B.perm : B.bin_order;
        const int lim = MODE == 0 ? B.nlocal : n_all(B);
        for (int b0 = U.begin + 4 * w; b0 < U.end; b0 += 32) {
            const int b = b0 + grp;
            int n = 0, s = 0;
            if (b < U.end) {
                n = cnt[b];
                s = start[b];
            }
            if (n != 0 && !(MDPD_IN(s, s + n) && MDPD_IN(s + n - 1, lim))) {
                if (l8 == 0) cnt[b] = 0;  // check build: a bucket outside its array
                n = 0;
            }
            if (MODE == 1) {
                // a bin whose last member is a local holds no ghost image (locals come first): it
                // is already in index order, its bpos written by the scatter
                int last = 0;
                if (n > 0 && l8 == 0) last = arr[s + n - 1];
                last = __shfl_sync(0xffffffffu, last, grp << 3);
                if (n > 0 && last < B.nlocal) {
                    if (l8 == 0) cnt[b] = 0;
                    n = 0;
                }
            }
            const bool group = n > 0 && n <= 8 * kGroupSlots;
            const int slots = __reduce_max_sync(0xffffffffu, group ? (n + 7) >> 3 : 0);  // warp-uniform
            int idx[kGroupSlots];
            unsigned long long k[kGroupSlots];
#pragma unroll
            for (int m = 0; m < kGroupSlots; ++m) {
                idx[m] = 0;
                if (group && l8 + 8 * m < n) idx[m] = MDPD_IDX(arr[s + l8 + 8 * m], lim);
            }
#pragma unroll
            for (int m = 0; m < kGroupSlots; ++m) {
                k[m] = ~0ull;  // no member: above every key, counted by no rank
                if (group && l8 + 8 * m < n)
                    k[m] = MODE == 0 ? (((unsigned long long)(uint32_t)B.sub_of[idx[m]] << 32) | (uint32_t)idx[m])
                                     : (unsigned long long)(uint32_t)idx[m];
            }
            // rank of each member: the group's keys below it (every member's key is loaded before
            // any lane gets past these shuffles, so the stores below cannot overwrite an unread one)
            int rank[kGroupSlots] = {};
#pragma unroll
            for (int mm = 0; mm < kGroupSlots; ++mm) {
                if (mm >= slots) break;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const unsigned long long kq = __shfl_sync(0xffffffffu, k[mm], (grp << 3) | q);
#pragma unroll
                    for (int m = 0; m < kGroupSlots; ++m) rank[m] += kq < k[m] ? 1 : 0;
                }
            }
#pragma unroll
            for (int m = 0; m < kGroupSlots; ++m) {
                if (group && l8 + 8 * m < n) {
                    arr[s + rank[m]] = idx[m];
                    if (MODE == 1) B.bpos[s + rank[m]] = list_pos(B.pos[idx[m]], idx[m], B.nlocal);
                }
            }
            if (group && l8 == 0) cnt[b] = 0;
            // buckets of more than 32 members: the whole warp, one after another
            unsigned big = __ballot_sync(0xffffffffu, l8 == 0 && n > 8 * kGroupSlots);
            while (big) {
                const int leader = __ffs(big) - 1;
                big &= big - 1;
                const int bb = b0 + (leader >> 3);
                const int nb = __shfl_sync(0xffffffffu, n, leader), sb = __shfl_sync(0xffffffffu, s, leader);
                __syncwarp();
                if (nb > kClassMax) {
                    if (lane == 0) atomicOr(&B.st->status, kErrBucketOverflow);
                } else
                    bucket_warp<MODE>(B, arr, sb, nb, lane, key);
                if (lane == 0) cnt[bb] = 0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// R5: permute into the other buffer; pack; ghost-image counts; bin the locals
// ---------------------------------------------------------------------------
__device__ __forceinline__ int image_mask(const BoxDesc &B, double x, int d)
{
    // bit 0: image at +prd (x within cutghost of lo), bit 1: image at -prd
    int m = 0;
    if (x <= B.lo[d] + B.cutghost) m |= 1;
    if (x >= B.hi[d] - B.cutghost) m |= 2;
    return m;
}

__device__ __forceinline__ int bits_count(int m) { return 1 + (m & 1) + ((m >> 1) & 1); }

template <int STYLE>
__global__ void __launch_bounds__(kUnit) k_rb_permute(BoxDesc *__restrict__ boxes,
                                                      const Unit *__restrict__ units, int nunits,
                                                      int nbox, int *done)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int k = U.begin + threadIdx.x;
        if (k >= U.end) continue;
        const BoxState &S = *B.st;
        const int c = S.cur, o = 1 - c;
        const int old = MDPD_IDX(B.perm[k], B.nlocal);
        // every load of the particle is issued before the first store (the compiler may not move
        // a load above a store to a possibly aliased array): one memory round trip
        double x[3], v[3];
        for (int d = 0; d < 3; ++d) {
            x[d] = B.x[c][d][old];
            v[d] = B.v[c][d][old];
        }
        const float4 f = B.f[c][old];
        const int tag = B.tag[c][old], type = B.type[c][old], mask = B.mask[c][old];
        const float phi = B.phi[c][old];
        // packed state for the current step (the step counter was advanced by integrate, which
        // left this step's seed in the box state)
        const long long step = S.step;
        const bool sn_cached = S.sn_ok && S.sn_step == step + 1 && S.sn_seed == B.seed;
        const uint32_t sn = sn_cached ? S.sn_prev : seed_now(B.seed, step);  // box-uniform branch
        for (int d = 0; d < 3; ++d) {
            B.x[o][d][k] = x[d];
            B.v[o][d][k] = v[d];
            B.xh[d][k] = x[d];
        }
        B.f[o][k] = f;
        B.tag[o][k] = tag;
        B.type[o][k] = type;
        B.mask[o][k] = mask;
        B.phi[o][k] = phi;
        const float fvx = (float)v[0], fvy = (float)v[1], fvz = (float)v[2];
        B.pos[k] = make_float4((float)(x[0] - B.cen[0]), (float)(x[1] - B.cen[1]),
                               (float)(x[2] - B.cen[2]), pack_w(B, type, mask));
        const uint32_t sg = STYLE == 0 ? sig_mdpd(tag, sn) : sig_dpd(tag, fvx, fvy, fvz, sn);
        B.vel[k] = make_float4(fvx, fvy, fvz, __uint_as_float(sg));
        // ghost images of this particle
        int nimg = 1;
        for (int d = 0; d < 3; ++d) nimg *= bits_count(image_mask(B, x[d], d));
        B.gfirst[k] = nimg - 1;
        if (k == B.nlocal - 1) B.gfirst[B.nlocal] = 0;
        // bin of the local
        int bid[3];
        for (int d = 0; d < 3; ++d) bid[d] = clamp_bin(bin_coord(x[d], B.lo[d], B.bininv[d]), B.mbin[d]);
        const int bin = bid[0] + B.mbin[0] * (bid[1] + bid[2] * B.mbin[1]);
        B.bin_of[k] = bin;
        warp_add1(B.bin_count, MDPD_IDX(bin, B.nbin));
    }
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        for (int b = threadIdx.x; b < nbox; b += blockDim.x) {
            BoxState *S = boxes[b].st;
            if (S->rebuild) {
                S->cur = 1 - S->cur;
                S->n_bulk = boxes[b].cls_start[boxes[b].nbin];
            }
        }
        if (threadIdx.x == 0) *done = 0;
    }
}

// ---------------------------------------------------------------------------
// R7: ghost images of border particles + their bins
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUnit) k_rb_ghosts(const BoxDesc *__restrict__ boxes,
                                                     const Unit *__restrict__ units, int nunits)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int k = U.begin + threadIdx.x;
        if (k >= U.end || k < B.st->n_bulk) continue;
        const int c = B.st->cur;
        const int g0 = B.gfirst[k], g1 = B.gfirst[k + 1];
        if (g1 == g0) continue;
        double x[3];
        int m[3];
        for (int d = 0; d < 3; ++d) {
            x[d] = B.x[c][d][k];
            m[d] = image_mask(B, x[d], d);
        }
        const float4 vk = B.vel[k];
        const float w = B.pos[k].w;
        int g = g0;
        for (int sz = -1; sz <= 1; ++sz) {
            if (sz == 1 && !(m[2] & 1)) continue;
            if (sz == -1 && !(m[2] & 2)) continue;
            for (int sy = -1; sy <= 1; ++sy) {
                if (sy == 1 && !(m[1] & 1)) continue;
                if (sy == -1 && !(m[1] & 2)) continue;
                for (int sx = -1; sx <= 1; ++sx) {
                    if (sx == 1 && !(m[0] & 1)) continue;
                    if (sx == -1 && !(m[0] & 2)) continue;
                    if (sx == 0 && sy == 0 && sz == 0) continue;
                    if (g >= B.ghost_cap) {
                        atomicOr(&B.st->status, kErrGhostOverflow);
                        continue;
                    }
                    const double gx = x[0] + sx * B.prd[0];
                    const double gy = x[1] + sy * B.prd[1];
                    const double gz = x[2] + sz * B.prd[2];
                    const int gi = B.nlocal + g;
                    B.gsrc[g] = k;
                    const int code = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1);
                    B.gimg[g] = code;
                    B.pos[gi] = make_float4((float)(gx - B.cen[0]), (float)(gy - B.cen[1]),
                                            (float)(gz - B.cen[2]), ghost_w(w, code));
                    B.vel[gi] = vk;
                    const double gc[3] = {gx, gy, gz};
                    int bid[3];
                    for (int d = 0; d < 3; ++d) {
                        const double v = gc[d];
                        const int b = clamp_bin(bin_coord(v, B.lo[d], B.bininv[d]), B.mbin[d]);
                        bid[d] = v >= B.lo[d] ? (v <= B.hi[d] ? b : B.mbin[d] - 1) : 0;
                    }
                    const int bin = bid[0] + B.mbin[0] * (bid[1] + bid[2] * B.mbin[1]);
                    B.bin_of[gi] = bin;
                    atomicAdd(&B.bin_count[MDPD_IDX(bin, B.nbin)], 1);
                    ++g;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// R9: scatter locals+ghosts into bins.  A local's place needs no atomics: the reorder sort
// left a bin's bulk particles, then its border particles, as two runs of consecutive indices,
// so its rank in the bin (in index order) follows from the class starts; its packed position
// goes to bpos as well.  Ghost images take atomic slots after the bin's locals, and the bin
// sort puts them in index order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kUnit) k_rb_scatter_bins(const BoxDesc *__restrict__ boxes,
                                                           const Unit *__restrict__ units, int nunits)
{
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const Unit U = units[u];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int i = U.begin + threadIdx.x;
        const int nl = B.nlocal;
        if (i >= U.end || i >= nl + min(B.st->nghost, B.ghost_cap)) continue;
        const int bin = MDPD_IDX(B.bin_of[i], B.nbin);
        const int rk = B.bin_rank[bin];
        const int b0 = B.cls_start[rk], b1 = B.cls_start[rk + 1];  // the bin's bulk run
        const int e0 = B.cls_start[B.nbin + rk];                     // its border run
        int p;
        if (i < nl) {
            p = MDPD_IDX(B.bin_start[bin] + (i < B.st->n_bulk ? i - b0 : (b1 - b0) + (i - e0)), n_all(B));
            B.bpos[p] = list_pos(B.pos[i], i, nl);
        } else {
            const int nloc = (b1 - b0) + (B.cls_start[B.nbin + rk + 1] - e0);
            p = MDPD_IDX(warp_add1(B.bin_cursor, bin) + nloc, n_all(B));
        }
        B.bin_order[p] = i;
    }
}

// ---------------------------------------------------------------------------
// R11: neighbour list, warp per bin, in two phases per chunk of candidates:
//   filter  the 27 stencil bins are streamed once (lane = candidate, its bin found from one
//           ballot and one OR-reduction of the bins' start offsets); a candidate is kept
//           when it lies within the cutoff of the box bounding the bin's centres (the FP32
//           bound is exact: each axis gap rounds to at most the gap to any centre, and the
//           squared distance is monotone in the gaps), compacted into shared memory
//           (x, y, z, list word; the particle index beside it).  On a reduced list a candidate
//           below every centre of the batch (a smaller local index or a lower ghost image) is
//           owned by none of them and can only be a hit within rn2_list, so it is kept only
//           within that radius of the box
//   test    two kept candidates per lane (k and k + 32 of a 64-candidate round), loop over the
//           centres; the squared distances of both come from one two-lane FP32 evaluation
//           (sub/mul/fma .f32x2, rounded per lane as the scalar dist2); the ballots of centre c
//           are its hits in the round, and each hit's lane writes it straight into c's row at
//           c's count plus its rank in the ballots, so rows fill in candidate order
// A hit is a pair within the cutoff, not the centre itself; on a box with list_reduce also
// owned by the centre (a local above it, or an upper ghost image) or within rn2_list: the
// other pairs can enter neither the density sum nor the pair-once force list before the next
// build.
// Work items are 8 bins (one per warp) of a 256-bin unit, taken grid-stride so every SM
// stays full whatever the number of rebuilding boxes.
// ---------------------------------------------------------------------------
constexpr int kListChunk = 224;                 // kept candidates per chunk (3.5 rounds)

__device__ __forceinline__ float warp_min(float v)
{
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_max(float v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// 4 blocks per SM: 64 registers
__global__ void __launch_bounds__(256, 4) k_rb_list(const BoxDesc *__restrict__ boxes,
                                                 const Unit *__restrict__ units, int nunits,
                                                 int nbox, int *done)
{
    __shared__ float4 s_ca[8][32], s_cb[8][32];         // centres: x, x, y, y | z, z, index, row offset
    __shared__ int s_n[8][32];                          // entries of each centre so far
    __shared__ float4 s_q[8][kListChunk];               // kept candidates: x, y, z, list word
    __shared__ int s_j[8][kListChunk];                  // their particle indices
    __shared__ float4 s_lo[8], s_hi[8];                 // the centres' bounding box; cmin
    __shared__ int s_d[8][32], s_ex[8][32];             // non-empty stencil bins: start - stream offset; offset
    const int lane = threadIdx.x & 31, w = threadIdx.x / 32;
    const unsigned lt = (1u << lane) - 1u;
    const int nitems = nunits * 32;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const Unit U = units[it >> 5];
        const BoxDesc &B = boxes[U.box];
        if (!rebuilding(B)) continue;
        const int b = U.begin + ((it & 31) << 3) + w;
        if (b >= U.end) continue;
        const int s = B.bin_start[b], e = B.bin_start[b + 1];
        if (e == s) continue;
        if (!(MDPD_IN(s, e) && MDPD_IN(e - 1, n_all(B)))) continue;  // check build: a bin outside the arrays
        if (B.bin_order[s] >= B.nlocal) continue;  // no locals in this bin
        const float rc2 = B.rc2_tail;
        const float rn2 = B.list_reduce ? B.rn2_list : rc2;  // with rc2: every pair (full list)
        // a row marks the entries its centre owns with bit 31 (kOwnedEntry), which the pair-once
        // density pass reads instead of re-deriving ownership per step; other readers mask it off
        const int own = (int)kOwnedEntry;
        const int ncol = B.n_col, nlocal = B.nlocal;
        int *const table = B.table;
        const int bx = b % B.mbin[0], by = (b / B.mbin[0]) % B.mbin[1], bz = b / (B.mbin[0] * B.mbin[1]);
        // stencil bins: lane l < 27 takes offset (l%3-1, l/3%3-1, l/9-1)
        int st = 0, sz = 0;
        if (lane < 27) {
            const int x = bx + lane % 3 - 1, y = by + (lane / 3) % 3 - 1, z = bz + lane / 9 - 1;
            if (x >= 0 && x < B.mbin[0] && y >= 0 && y < B.mbin[1] && z >= 0 && z < B.mbin[2]) {
                const int nb = x + B.mbin[0] * (y + z * B.mbin[1]);
                st = B.bin_start[nb];
                sz = B.bin_start[nb + 1] - st;
                if (sz != 0 && !(MDPD_IN(st, st + sz) && MDPD_IN(st + sz - 1, n_all(B)))) sz = 0;
            }
        }
        int cum = sz;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, cum, o);
            if (lane >= o) cum += v;
        }
        const int total = __shfl_sync(0xffffffffu, cum, 31);
        // the candidate stream is the non-empty stencil bins in slot order; bin k of them starts
        // at stream offset ex_k, so stream position q is particle d_k + q of the bin order with
        // d_k = start_k - ex_k, k the last non-empty bin with ex_k <= q
        const unsigned ne = __ballot_sync(0xffffffffu, sz != 0);
        if (sz != 0) {
            const int k = __popc(ne & lt);
            s_d[w][k] = st - (cum - sz);
            s_ex[w][k] = cum - sz;
        }
        __syncwarp();
        // lane k holds ex_k of non-empty bin k (no bin: past every position)
        const int exk = lane < __popc(ne) ? s_ex[w][lane] : 0x7fffffff;
        const unsigned le = lt | (1u << lane);
        int local_max = 0;
        for (int cb = s; cb < e; cb += 32) {
            // centre batch: members with index < nlocal (they come first in a bin)
            const int pc = cb + lane;
            const int ci = pc < e ? MDPD_IDX(B.bin_order[pc], n_all(B)) : nlocal;
            const bool is_c = ci < nlocal;
            const unsigned cm = __ballot_sync(0xffffffffu, is_c);
            if (cm == 0) break;
            const int nc = __popc(cm);
            const float4 pc4 = is_c ? B.bpos[pc] : make_float4(0.f, 0.f, 0.f, 0.f);
            s_ca[w][lane] = make_float4(pc4.x, pc4.x, pc4.y, pc4.y);
            // entry p of centre i at (i & ~31) * ncol + 32 p + (i & 31): entries p of 32
            // consecutive centres are contiguous
            s_cb[w][lane] = make_float4(pc4.z, pc4.z, __int_as_float(ci),
                                        __uint_as_float((unsigned)(ci & ~31) * (unsigned)ncol + (unsigned)(ci & 31)));
            s_n[w][lane] = 0;
            {
                const float inf = __int_as_float(0x7f800000);
                const float lox = warp_min(is_c ? pc4.x : inf), hix = warp_max(is_c ? pc4.x : -inf);
                const float loy = warp_min(is_c ? pc4.y : inf), hiy = warp_max(is_c ? pc4.y : -inf);
                const float loz = warp_min(is_c ? pc4.z : inf), hiz = warp_max(is_c ? pc4.z : -inf);
                // smallest centre index of the batch: a candidate below it (a local with a smaller
                // index, or a lower ghost image) is owned by none of the centres, so on a reduced
                // list it is a hit only within rn2, and the filter keeps it only within rn2 of the box
                int cmin = is_c ? ci : 0x7fffffff;
                for (int o = 16; o > 0; o >>= 1) cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
                if (lane == 0) {
                    s_lo[w] = make_float4(lox, loy, loz, __int_as_float(cmin));
                    s_hi[w] = make_float4(hix, hiy, hiz, 0.f);
                }
            }
            __syncwarp();
            for (int qs = 0; qs < total;) {
                // filter: fill up to kListChunk kept candidates
                int nk = 0;
                const float4 lo = s_lo[w], hi = s_hi[w];
                for (; qs < total && nk <= kListChunk - 32; qs += 32) {
                    const int q = qs + lane;
                    // bin of position q: the bins that start before qs, plus those that start
                    // in [qs, q] (bit ex_k - qs of the round's start mask)
                    const unsigned starts = __reduce_or_sync(
                        0xffffffffu, exk >= qs && exk - qs < 32 ? 1u << (exk - qs) : 0u);
                    const int kq = __popc(__ballot_sync(0xffffffffu, exk < qs)) + __popc(starts & le) - 1;
                    bool keep = false;
                    float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (q < total) {
                        pj = B.bpos[s_d[w][kq] + q];
                        const float gx = fmaxf(fmaxf(lo.x - pj.x, pj.x - hi.x), 0.f);
                        const float gy = fmaxf(fmaxf(lo.y - pj.y, pj.y - hi.y), 0.f);
                        const float gz = fmaxf(fmaxf(lo.z - pj.z, pj.z - hi.z), 0.f);
                        keep = dist2(gx, gy, gz) <= (__float_as_int(pj.w) < __float_as_int(lo.w) ? rn2 : rc2);
                    }
                    const unsigned kb = __ballot_sync(0xffffffffu, keep);
                    if (keep) {
                        const int k = nk + __popc(kb & lt);
                        const int wd = __float_as_int(pj.w);
                        s_q[w][k] = pj;
                        s_j[w][k] = MDPD_IDX(wd ^ (wd >> 31), n_all(B));
                    }
                    nk += __popc(kb);
                }
                __syncwarp();
                for (int r0 = 0; r0 < nk; r0 += 64) {
                    const int ka = r0 + lane, kb2 = ka + 32;
                    const float4 pa = ka < nk ? s_q[w][ka] : make_float4(1e30f, 1e30f, 1e30f, 0.f);
                    const float4 pb = kb2 < nk ? s_q[w][kb2] : make_float4(1e30f, 1e30f, 1e30f, 0.f);
                    const int ja = ka < nk ? s_j[w][ka] : 0, jb = kb2 < nk ? s_j[w][kb2] : 0;
                    const int wa = __float_as_int(pa.w), wb = __float_as_int(pb.w);
                    const unsigned long long px = pk2(pa.x, pb.x), py = pk2(pa.y, pb.y), pz = pk2(pa.z, pb.z);
#pragma unroll 1
                    for (int c = 0; c < nc; ++c) {
                        const float4 A = s_ca[w][c], C = s_cb[w][c];
                        const int cic = __float_as_int(C.z);
                        float r2a, r2b;
                        upk2(dist2x2(sub2(pk2(A.x, A.y), px), sub2(pk2(A.z, A.w), py), sub2(pk2(C.x, C.y), pz)),
                             r2a, r2b);
                        // owned candidates are hits within rc2, the others within rn2 (<= rc2)
                        const bool oa = wa > cic, ob = wb > cic;
                        const bool ha = r2a <= (oa ? rc2 : rn2) && wa != cic;
                        const bool hb = r2b <= (ob ? rc2 : rn2) && wb != cic;
                        const unsigned bala = __ballot_sync(0xffffffffu, ha);
                        const unsigned balb = __ballot_sync(0xffffffffu, hb);
                        const int n0 = s_n[w][c];
                        const int na = n0 + __popc(bala);
                        // a row that would overflow keeps writing its last entry (the count
                        // reports the overflow); the table holds ncol entries per row
                        const unsigned row = __float_as_uint(C.w);
                        if (ha)
                            table[row + 32u * (unsigned)min(n0 + __popc(bala & lt), ncol - 1)] = ja | (oa ? own : 0);
                        if (hb)
                            table[row + 32u * (unsigned)min(na + __popc(balb & lt), ncol - 1)] = jb | (ob ? own : 0);
                        s_n[w][c] = na + __popc(balb);  // every lane stores the same count
                    }
                }
                __syncwarp();
            }
            if (is_c) {
                const int my_n = s_n[w][lane];
                B.count[ci] = my_n < ncol ? my_n : ncol;
                if (my_n > ncol) atomicOr(&B.st->status, kErrListOverflow);
                local_max = max(local_max, my_n);
            }
            __syncwarp();
        }
        for (int o = 16; o > 0; o >>= 1) local_max = max(local_max, __shfl_xor_sync(0xffffffffu, local_max, o));
        if (lane == 0 && local_max > 0) atomicMax(&B.st->max_count, local_max);
    }
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        for (int b = threadIdx.x; b < nbox; b += blockDim.x) {
            BoxState *S = boxes[b].st;
            if (S->rebuild) S->nbuild += 1;
        }
        if (threadIdx.x == 0) *done = 0;
    }
}

__global__ void k_bin_ranks(int mx, int my, int mz, int *rank)
{
    const int nbin = mx * my * mz;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbin; b += gridDim.x * blockDim.x)
        rank[b] = morton_rank(b % mx, (b / mx) % my, b / (mx * my), mx, my, mz);
}

void launch_bin_ranks(cudaStream_t s, const int mbin[3], int *rank)
{
    const int nbin = mbin[0] * mbin[1] * mbin[2];
    k_bin_ranks<<<std::min((nbin + 255) / 256, 148 * 8), 256, 0, s>>>(mbin[0], mbin[1], mbin[2], rank);
}

// Resident blocks per SM of the per-particle rebuild passes (kUnit threads each). They loop over
// units one particle per thread, waiting on each unit's loads, so they run as fast as the SM
// holds blocks: the grid is the occupancy the registers allow (12 to 16 blocks for the lighter
// passes), not a fixed 8.
struct RebuildShapes {
    int key = 8, cls = 8, permute0 = 8, permute1 = 8, ghosts = 8, bins = 8;
};
static RebuildShapes g_shapes;
static std::once_flag g_shapes_once;

template <typename K> static int resident_blocks(K kernel, int threads = kUnit, int fallback = 8)
{
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, 0) != cudaSuccess || b < 1) {
        (void)cudaGetLastError();  // a failed query leaves the fixed grid
        return fallback;
    }
    return b;
}

void init_rebuild_shapes()
{
    std::call_once(g_shapes_once, [] {
        g_shapes.key = resident_blocks(k_rb_key);
        g_shapes.cls = resident_blocks(k_rb_scatter_cls);
        g_shapes.permute0 = resident_blocks(k_rb_permute<0>);
        g_shapes.permute1 = resident_blocks(k_rb_permute<1>);
        g_shapes.ghosts = resident_blocks(k_rb_ghosts);
        g_shapes.bins = resident_blocks(k_rb_scatter_bins);
        g_scan_reduce[0] = resident_blocks(k_scan_reduce<0>, 256, 4);
        g_scan_reduce[1] = resident_blocks(k_scan_reduce<1>, 256, 4);
        g_scan_reduce[2] = resident_blocks(k_scan_reduce<2>, 256, 4);
        g_scan_down[0] = resident_blocks(k_scan_down<0>, 256, 4);
        g_scan_down[1] = resident_blocks(k_scan_down<1>, 256, 4);
        g_scan_down[2] = resident_blocks(k_scan_down<2>, 256, 4);
    });
}

void launch_rebuild(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int *done)
{
    init_rebuild_shapes();  // a no-op after the first call (made before any capture)
    const int sms = c.sms;
    const RebuildShapes &r = g_shapes;
    auto g = [&](int n, int per_sm) { return n < sms * per_sm ? (n > 0 ? n : 1) : sms * per_sm; };
    k_rb_key<<<g(u.local.n, r.key), kUnit, 0, s>>>(boxes, u.local.d, u.local.n);
    scan<kSelCls>(s, boxes, u.scan_cls, u.nbox, sms);
    k_rb_scatter_cls<<<g(u.local.n, r.cls), kUnit, 0, s>>>(boxes, u.local.d, u.local.n);
    k_rb_bucket<0><<<g(u.cls.n, 4), 256, 0, s>>>(boxes, u.cls.d, u.cls.n);
    if (c.style == 0)
        k_rb_permute<0><<<g(u.local.n, r.permute0), kUnit, 0, s>>>(boxes, u.local.d, u.local.n, u.nbox, done);
    else
        k_rb_permute<1><<<g(u.local.n, r.permute1), kUnit, 0, s>>>(boxes, u.local.d, u.local.n, u.nbox, done);
    scan<kSelGhost>(s, boxes, u.scan_ghost, u.nbox, sms);
    k_rb_ghosts<<<g(u.local.n, r.ghosts), kUnit, 0, s>>>(boxes, u.local.d, u.local.n);
    scan<kSelBin>(s, boxes, u.scan_bin, u.nbox, sms);
    k_rb_scatter_bins<<<g(u.all.n, r.bins), kUnit, 0, s>>>(boxes, u.all.d, u.all.n);
    k_rb_bucket<1><<<g(u.bins.n, 4), 256, 0, s>>>(boxes, u.bins.d, u.bins.n);
    k_rb_list<<<g(u.bins.n * 32, 4), 256, 0, s>>>(boxes, u.bins.d, u.bins.n, u.nbox, done + 1);
}

}  // namespace mdpd
