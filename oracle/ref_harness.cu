/*
 * Reference harness -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 *   ref_harness <case.bin> <out.bin>
 *
 * Runs the reference's own device kernels of the rebuild and pair path on one periodic box
 * read from <case.bin> and writes what they produce to <out.bin>.  The reference sources below
 * are compiled unmodified from the reference tree (build recipe: the `harness` target of
 * oracle/Makefile); only this driver is ours.  Kernels driven, in the order of a reference
 * rebuild and force evaluation (ModifiedVerlet::run, mvv_meso.cu:336-402, pre_force and
 * pair compute):
 *   gpu_build_reorder_keypair<1>              atom_meso.cu:271-311   (MesoAtom::sort_local :346-387)
 *   gpu_radix_histogram/prefix_sum/permute    sort_meso.h:21-106     (SortPlan::sort :384-406)
 *   gpu_assign_bin_id, gpu_find_bin_boundary,
 *   gpu_calc_bin_size, gpu_expand_stencil     neighbor_meso.cu:390-514 (binning_meso :539-660)
 *   gpu_stencil_full_bin_3d                   neighbor_meso.cu:685-738 (:740-769)
 *   gpu_merge_xvt_mdpd                        atom_vec_mdpd_atomic_meso.cu:140-206
 *   gpu_build_neighbor_list<32,5>, gpu_join_neigh_list, gpu_transpose_neigh_list
 *                                             neigh_build_meso.cu:17-127,188-272 (full_bin_meso :286-380)
 *   gpu_compute_rho                           fix_aboundary_rho_meso.cu:119-165 (pre_force :167-212)
 *   gpu_aboundary                             fix_aboundary_rho_meso.cu:220-287 (wall cases)
 *   gpu_mdpd<1>                               pair_mdpd_meso.cu:93-228 (compute_kernel :230-261)
 *
 * Host-side glue of the reference that needs the LAMMPS core objects is restated here instead
 * (these feed the kernels; they are not the pinned results): the bin geometry of
 * MesoNeighbor::setup_bins (neighbor_meso.cu:771-853), the slab bounds of Comm::setup
 * (comm.cpp:573-628) with MesoComm::borderness (comm_meso.cu:195-261), the periodic ghost
 * images of MesoComm::borders (comm_meso.cu:42-193) with pack_border_vel, the list sizes of
 * MesoNeighList (neigh_list_meso.cu:78-103), the forward communication of ghost rho
 * (fix_aboundary_rho_meso.cu:191-210) and the launch shapes.
 */
#include "neighbor_meso.cu"
#include "neigh_build_meso.cu"
#include "atom_meso.cu"
#include "fix_aboundary_rho_meso.cu"
#include "pair_mdpd_meso.cu"
#include "atom_vec_mdpd_atomic_meso.cu"
#include "sort_meso.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace LAMMPS_NS;

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #call, cudaGetErrorString(e_));   \
            exit(3);                                                                                 \
        }                                                                                            \
    } while (0)

static void fail(const char *msg)
{
    fprintf(stderr, "ref_harness: %s\n", msg);
    exit(2);
}

// ------------------------------------------------------------------ case file
struct Case {
    int n, ntype, arb_bc;
    double lo[3], hi[3];
    double cutforce, skin, rho_est, dt;
    double cut_rho, cut_phi, rho_wall, phi_c;
    uint32_t seed;
    int64_t step;
    int rho_bit, mobile_bit, wall_bit;
    double mass[8];
    std::vector<double> coeff;  // ntype*ntype*6: cut, cut_r, A, B, gamma, sigma
    std::vector<double> x[3], v[3];
    std::vector<int> tag, type, mask;
};

template <class T> static void rd(FILE *f, T *p, size_t n)
{
    if (n && fread(p, sizeof(T), n, f) != n) fail("short case file");
}

static Case read_case(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) fail("cannot open case file");
    char magic[8];
    rd(f, magic, 8);
    if (memcmp(magic, "MDPDCASE", 8)) fail("bad case magic");
    Case c;
    int pad;
    rd(f, &c.n, 1), rd(f, &c.ntype, 1), rd(f, &c.arb_bc, 1), rd(f, &pad, 1);
    rd(f, c.lo, 3), rd(f, c.hi, 3);
    rd(f, &c.cutforce, 1), rd(f, &c.skin, 1), rd(f, &c.rho_est, 1), rd(f, &c.dt, 1);
    rd(f, &c.cut_rho, 1), rd(f, &c.cut_phi, 1), rd(f, &c.rho_wall, 1), rd(f, &c.phi_c, 1);
    rd(f, &c.seed, 1), rd(f, &pad, 1), rd(f, &c.step, 1);
    rd(f, &c.rho_bit, 1), rd(f, &c.mobile_bit, 1), rd(f, &c.wall_bit, 1), rd(f, &pad, 1);
    rd(f, c.mass, 8);
    if (c.n < 1 || c.n > 4000000 || c.ntype < 1 || c.ntype > 8) fail("case sizes out of range");
    c.coeff.resize((size_t)c.ntype * c.ntype * 6);
    rd(f, c.coeff.data(), c.coeff.size());
    for (int d = 0; d < 3; ++d) c.x[d].resize(c.n), rd(f, c.x[d].data(), c.n);
    for (int d = 0; d < 3; ++d) c.v[d].resize(c.n), rd(f, c.v[d].data(), c.n);
    c.tag.resize(c.n), c.type.resize(c.n), c.mask.resize(c.n);
    rd(f, c.tag.data(), c.n), rd(f, c.type.data(), c.n), rd(f, c.mask.data(), c.n);
    fclose(f);
    for (int i = 0; i < c.n; ++i) {
        if (c.type[i] < 1 || c.type[i] > c.ntype) fail("atom type out of range");
        for (int d = 0; d < 3; ++d)
            if (!(c.x[d][i] >= c.lo[d] && c.x[d][i] < c.hi[d])) fail("position outside the box");
    }
    return c;
}

// ------------------------------------------------------------------ output file
struct Out {
    FILE *f;
    explicit Out(const char *path) : f(fopen(path, "wb"))
    {
        if (!f) fail("cannot open output");
    }
    ~Out() { fclose(f); }
    template <class T> void put(const char *name, const char *dtype, const T *p, int64_t n)
    {
        char nm[32] = {0}, dt[8] = {0};
        strncpy(nm, name, 31);
        strncpy(dt, dtype, 7);
        fwrite(nm, 1, 32, f);
        fwrite(dt, 1, 8, f);
        fwrite(&n, sizeof(n), 1, f);
        if (n) fwrite(p, sizeof(T), (size_t)n, f);
    }
};

template <class T> struct Dev {
    T *p = nullptr;
    size_t n = 0;
    explicit Dev(size_t n_ = 0) { alloc(n_); }
    void alloc(size_t n_)
    {
        if (p) cudaFree(p);
        n = n_ ? n_ : 1;
        CK(cudaMalloc(&p, n * sizeof(T)));
        CK(cudaMemset(p, 0, n * sizeof(T)));
    }
    ~Dev()
    {
        if (p) cudaFree(p);
    }
    void up(const T *h, size_t m)
    {
        if (m > n) fail("upload larger than its buffer");
        CK(cudaMemcpy(p, h, m * sizeof(T), cudaMemcpyHostToDevice));
    }
    std::vector<T> down(size_t m) const
    {
        if (m > n) fail("download larger than its buffer");
        std::vector<T> h(m);
        CK(cudaMemcpy(h.data(), p, m * sizeof(T), cudaMemcpyDeviceToHost));
        return h;
    }
};

static cudaTextureObject_t linear_tex(void *ptr, size_t bytes, cudaChannelFormatDesc desc)
{
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = ptr;
    rd.res.linear.desc = desc;
    rd.res.linear.sizeInBytes = bytes;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t t;
    CK(cudaCreateTextureObject(&t, &rd, &td, nullptr));
    return t;
}

// SortPlan<16,K,V>::sort (sort_meso.h:384-406) with the reference's own pass kernels; the
// histogram and permute kernels are grid-stride loops and the prefix sum runs one block per
// radix digit, so the launch shape below (any multiple of 32 threads) gives the same result
template <class K> static void radix_sort(Dev<K> &key, Dev<int> &val, int n, int n_bit)
{
    const int RADIX = 16;
    const int warp_padding = (n + WARPSZ - 1) / WARPSZ + 1;
    Dev<K> key_out(n);
    Dev<int> val_out(n), tprev(n), wprev((size_t)warp_padding * RADIX);
    K *kin = key.p, *kout = key_out.p;
    int *vin = val.p, *vout = val_out.p;
    const int blocks = std::max(1, std::min(1184, (n + 255) / 256));
    for (int bit = 0; bit < n_bit; bit += 4) {
        gpu_radix_histogram<RADIX, K><<<blocks, 256>>>(kin, tprev.p, wprev.p, n, bit, warp_padding);
        gpu_radix_prefix_sum<int><<<RADIX, 1024>>>(wprev.p, (n + WARPSZ - 1) / WARPSZ, warp_padding);
        gpu_radix_permute<RADIX, K, int><<<blocks, 256>>>(kin, vin, kout, vout, tprev.p, wprev.p, n, bit,
                                                          warp_padding);
        CK(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    if (kin != key.p) {
        CK(cudaMemcpy(key.p, kin, n * sizeof(K), cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(val.p, vin, n * sizeof(int), cudaMemcpyDeviceToDevice));
    }
    CK(cudaDeviceSynchronize());
}

int main(int argc, char **argv)
{
    if (argc != 3) fail("usage: ref_harness <case.bin> <out.bin>");
    Case c = read_case(argv[1]);
    const int n = c.n;
    Out out(argv[2]);

    // ---- bin geometry: MesoNeighbor::setup_bins (neighbor_meso.cu:771-853) on one proc ----
    const double cutneighmax = c.cutforce + c.skin;  // Neighbor::init (neighbor.cpp:258-268)
    const double cutghost = cutneighmax;             // Comm::init (comm.cpp:413-415)
    double prd[3], bininv[3], binsize[3], cen[3];
    int mbin[3];
    for (int d = 0; d < 3; ++d) {
        prd[d] = c.hi[d] - c.lo[d];
        if (prd[d] < cutghost) fail("box side below the ghost cutoff (more than one swap per dim)");
        int nb = std::max((int)(prd[d] * (1.0 / cutneighmax)), 1);
        mbin[d] = nb + 2;
        binsize[d] = prd[d] / (mbin[d] - 2);
        bininv[d] = 1.0 / binsize[d];
        cen[d] = 0.5 * (c.hi[d] + c.lo[d]);  // dp2sp_merged offset (atom_vec_mdpd_atomic_meso.cu:180-184)
    }
    const int nbin = mbin[0] * mbin[1] * mbin[2];
    const double vol = prd[0] * prd[1] * prd[2];
    const double density = c.rho_est > 0 ? c.rho_est : n / vol;
    double expected_neigh = std::max(density * (4.0 / 3.0 * 3.142 * pow(cutneighmax, 3.0)) * 4.0, 32.0);
    const double expected_bin_size = density * cutneighmax * cutneighmax * cutneighmax;
    const int n_col = (((int)expected_neigh + 31) / 32) * 32;  // neigh_list_meso.cu:84 (ceiling to 32)

    // ---- borderness: slabs of Comm::setup (comm.cpp:573-628), counted per MesoComm::borderness ----
    const double kBig = 1.0e20;
    double slablo[6], slabhi[6];
    for (int d = 0; d < 3; ++d) {
        slablo[2 * d] = -kBig, slabhi[2 * d] = c.lo[d] + cutghost;
        slablo[2 * d + 1] = c.hi[d] - cutghost, slabhi[2 * d + 1] = kBig;
    }
    std::vector<int> border(n, 0);
    for (int i = 0; i < n; ++i)
        for (int s = 0; s < 6; ++s)
            if (c.x[s / 2][i] >= slablo[s] && c.x[s / 2][i] <= slabhi[s]) border[i]++;

    // ---- reorder keys + stable radix sort (MesoAtom::sort_local, atom_meso.cu:346-387) ----
    const int l2_resoln = 16;
    const int max_bin = std::max(std::max(mbin[0], mbin[1]), mbin[2]);
    const int l0_width = 1;
    const int l1_width = 3 * (int)floor(log2(max_bin * 2.0));
    const int l2_width = (int)(3 * log2((double)l2_resoln));
    const int l0_shift = l2_width + l1_width, l1_shift = l2_width, l2_shift = 0;
    const u64 border_mask = 1ULL << l0_shift;
    Dev<double> dx(n), dy(n), dz(n);
    dx.up(c.x[0].data(), n), dy.up(c.x[1].data(), n), dz.up(c.x[2].data(), n);
    Dev<u64> key(n);
    Dev<int> perm(n), dborder(n);
    dborder.up(border.data(), n);
    gpu_build_reorder_keypair<1><<<(n + 127) / 128, 128>>>(
        dx.p, dy.p, dz.p, key.p, perm.p, dborder.p, make_double3(c.lo[0], c.lo[1], c.lo[2]),
        make_double3(c.hi[0], c.hi[1], c.hi[2]), make_double3(bininv[0], bininv[1], bininv[2]),
        make_double3(l2_resoln * bininv[0], l2_resoln * bininv[1], l2_resoln * bininv[2]),
        make_double3(binsize[0], binsize[1], binsize[2]), make_int3(mbin[0], mbin[1], mbin[2]), l2_resoln,
        l1_shift, l2_shift, border_mask, n);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    std::vector<u64> key_unsorted = key.down(n);
    radix_sort<u64>(key, perm, n, l0_width + l1_width + l2_width);
    std::vector<int> p = perm.down(n);
    out.put("reorder_key", "u8", key_unsorted.data(), n);
    out.put("perm", "i4", p.data(), n);
    out.put("border", "i4", border.data(), n);

    // ---- apply the permutation (transfer_post_sort, atom_meso.cu:177-186) ----
    std::vector<double> X[3], V[3];
    std::vector<int> tag(n), type(n), mask(n), brd(n);
    for (int d = 0; d < 3; ++d) X[d].resize(n), V[d].resize(n);
    {
        std::vector<char> seen(n, 0);
        for (int i = 0; i < n; ++i) {
            const int s = p[i];
            if (s < 0 || s >= n || seen[s]) fail("sort output is not a permutation");
            seen[s] = 1;
            for (int d = 0; d < 3; ++d) X[d][i] = c.x[d][s], V[d][i] = c.v[d][s];
            tag[i] = c.tag[s], type[i] = c.type[s], mask[i] = c.mask[s], brd[i] = border[s];
        }
    }
    int n_bulk = 0;
    while (n_bulk < n && brd[n_bulk] == 0) ++n_bulk;
    for (int i = n_bulk; i < n; ++i)
        if (!brd[i]) fail("bulk particle after a border particle");

    // ---- periodic ghost images: MesoComm::borders (comm_meso.cu:42-193) on one proc ----
    // swap 2d sends slab [-BIG, lo+cutghost] shifted by +prd, swap 2d+1 sends
    // [hi-cutghost, BIG] shifted by -prd (pbc of comm.cpp:595-623); candidates of a dim are
    // [n_bulk, nlocal+nghost at the dim's first swap), in index order (pick_border)
    std::vector<int> gsrc, gimg;  // source local, image code (sx+1)+3(sy+1)+9(sz+1)
    for (int d = 0; d < 3; ++d) {
        const int nfirst = n_bulk, nlast = n + (int)gsrc.size();
        for (int side = 0; side < 2; ++side) {
            const double lo = slablo[2 * d + side], hi = slabhi[2 * d + side];
            const int shift = side == 0 ? 1 : -1;
            std::vector<int> add_src, add_img;
            for (int i = nfirst; i < nlast; ++i) {
                const int s = i < n ? i : gsrc[i - n];
                const int im = i < n ? 13 : gimg[i - n];
                const int sh[3] = {im % 3 - 1, (im / 3) % 3 - 1, im / 9 - 1};
                const double xd = X[d][s] + sh[d] * prd[d];
                if (xd >= lo && xd <= hi) {
                    int sn[3] = {sh[0], sh[1], sh[2]};
                    sn[d] += shift;
                    add_src.push_back(s);
                    add_img.push_back((sn[0] + 1) + 3 * (sn[1] + 1) + 9 * (sn[2] + 1));
                }
            }
            gsrc.insert(gsrc.end(), add_src.begin(), add_src.end());
            gimg.insert(gimg.end(), add_img.begin(), add_img.end());
        }
    }
    const int ng = (int)gsrc.size(), nall = n + ng;
    // ghost state: x + pbc*prd (pack_border_vel), v, tag, type, mask of the source
    for (int d = 0; d < 3; ++d) X[d].resize(nall), V[d].resize(nall);
    tag.resize(nall), type.resize(nall), mask.resize(nall);
    for (int g = 0; g < ng; ++g) {
        const int s = gsrc[g], im = gimg[g];
        const int sh[3] = {im % 3 - 1, (im / 3) % 3 - 1, im / 9 - 1};
        for (int d = 0; d < 3; ++d) X[d][n + g] = X[d][s] + sh[d] * prd[d], V[d][n + g] = V[d][s];
        tag[n + g] = tag[s], type[n + g] = type[s], mask[n + g] = mask[s];
    }
    out.put("ghost_src", "i4", gsrc.data(), ng);
    out.put("ghost_img", "i4", gimg.data(), ng);
    out.put("tag_all", "i4", tag.data(), nall);

    Dev<double> ax(nall), ay(nall), az(nall), avx(nall), avy(nall), avz(nall), amass(nall);
    Dev<int> atype(nall), atag(nall), amask(nall);
    ax.up(X[0].data(), nall), ay.up(X[1].data(), nall), az.up(X[2].data(), nall);
    avx.up(V[0].data(), nall), avy.up(V[1].data(), nall), avz.up(V[2].data(), nall);
    atype.up(type.data(), nall), atag.up(tag.data(), nall), amask.up(mask.data(), nall);
    {
        std::vector<double> m(nall);
        for (int i = 0; i < nall; ++i) m[i] = c.mass[type[i] - 1];  // per-atom mass (atom_vec_meso.h:216-230)
        amass.up(m.data(), nall);
    }

    // ---- binning: MesoNeighbor::binning_meso (neighbor_meso.cu:539-660) ----
    Dev<unsigned> bin_id(nall);
    Dev<int> atm_id(nall), bin_loc(nbin + 1), bin_isghost(nbin + 1), bin_size(nbin), bin_size_local(nbin);
    gpu_assign_bin_id<<<(nall + 127) / 128, 128>>>(ax.p, ay.p, az.p, bin_id.p, atm_id.p,
                                                   make_double3(c.lo[0], c.lo[1], c.lo[2]),
                                                   make_double3(c.hi[0], c.hi[1], c.hi[2]), mbin[0], mbin[1], mbin[2],
                                                   bininv[0], bininv[1], bininv[2], n, nall);
    CK(cudaGetLastError());
    const int bin_id_width = (int)ceil(log2((double)nbin));
    radix_sort<unsigned>(bin_id, atm_id, nall, bin_id_width);
    {
        // every bin id must lie in [0, nbin) before the boundary kernel indexes with it
        std::vector<unsigned> b = bin_id.down(nall);
        for (int i = 0; i < nall; ++i)
            if (b[i] >= (unsigned)nbin) fail("bin id out of range");
    }
    gpu_find_bin_boundary<<<(nall + 127) / 128, 128>>>(bin_id.p, atm_id.p, bin_loc.p, bin_isghost.p, nbin, n, nall);
    gpu_calc_bin_size<<<(nbin + 127) / 128, 128>>>(bin_loc.p, bin_isghost.p, bin_size.p, bin_size_local.p, nbin);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());

    // ---- stencil: stencil_full_bin_3d_meso (neighbor_meso.cu:740-769) + gpu_expand_stencil ----
    const int binsize_optimal = (int)cutneighmax;  // the reference truncates the cutoff to int here
    if (binsize_optimal < 1) fail("cutneighmax below 1");
    const int neighbor_range = (int)floor(cutneighmax / binsize_optimal + 0.5);
    const int side = 2 * neighbor_range + 1;
    const int nb_pad = ((side * side * side + 31) / 32) * 32;
    Dev<int> nb_count(nbin), nb_bin((size_t)nbin * nb_pad);
    Dev<unsigned long long> nb_key((size_t)nbin * nb_pad);
    {
        dim3 blk(8, 8, 8), grd((mbin[0] + 7) / 8, (mbin[1] + 7) / 8, (mbin[2] + 7) / 8);
        gpu_stencil_full_bin_3d<<<grd, blk>>>(nb_count.p, nb_bin.p, nb_key.p, mbin[0], mbin[1], mbin[2], neighbor_range,
                                              nb_pad);
        CK(cudaGetLastError());
    }
    std::vector<int> loc = bin_loc.down(nbin + 1), bsl = bin_size_local.down(nbin), nbc = nb_count.down(nbin);
    std::vector<int> nbb = nb_bin.down((size_t)nbin * nb_pad);
    int stencil_max = 0;
    for (int b = 0; b < nbin; ++b) {
        if (!bsl[b]) continue;
        int s = 0;
        for (int k = 0; k < nbc[b]; ++k) {
            const int nbn = nbb[(size_t)b * nb_pad + k];
            if (nbn < 0 || nbn >= nbin) fail("stencil bin out of range");
            s += loc[nbn + 1] - loc[nbn];
        }
        stencil_max = std::max(stencil_max, s);
    }
    const int stencil_pad = ((stencil_max + 31) / 32) * 32 + 32;
    Dev<int> stencil((size_t)nbin * stencil_pad), stencil_len(nbin);
    {
        const int tuple_size = std::max(8, (int)pow(2.0, (int)log2(expected_bin_size / 4)));
        if (tuple_size > 128 || 128 % tuple_size) fail("stencil tuple size does not divide the block");
        const long long threads = (long long)nbin * tuple_size;
        gpu_expand_stencil<<<(int)((threads + 127) / 128), 128>>>(atm_id.p, bin_loc.p, bin_size_local.p, nb_count.p,
                                                                 nb_bin.p, stencil.p, stencil_len.p, nb_pad,
                                                                 stencil_pad, tuple_size, nbin);
        CK(cudaGetLastError());
    }

    // ---- FP32 packing: dp2sp_merged with the step's seed (pair compute, pair_mdpd_meso.cu:287-297) ----
    uint32_t seed_now = premix_TEA<64>(c.seed, (uint)c.step);
    Dev<float4> coord(nall), veloc(nall);
    Dev<double> rho(nall);
    gpu_merge_xvt_mdpd<<<(nall + 127) / 128, 128>>>(ax.p, ay.p, az.p, avx.p, avy.p, avz.p, atype.p, atag.p, amass.p,
                                                    rho.p, coord.p, veloc.p, cen[0], cen[1], cen[2], (int)seed_now,
                                                    (int)(seed_now * 1664525U + 1013904223U), 0, nall);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    {
        std::vector<float4> pc = coord.down(nall), vc = veloc.down(nall);
        out.put("coord_merged", "f4", (const float *)pc.data(), 4LL * nall);
        out.put("veloc_merged", "f4", (const float *)vc.data(), 4LL * nall);
    }

    // ---- neighbour list: full_bin_meso (neigh_build_meso.cu:286-380) ----
    // rows for every particle, ghosts included: a local rounded into the outer bin layer makes
    // that bin a centre bin, whose ghosts then become rows too
    const int n_row = ((nall + 31) / 32) * 32;
    // guard regions before and after the table keep even an overflowing row inside the
    // allocation; an overflow is reported below and fails the case
    const size_t guard = (size_t)stencil_pad + 64;
    Dev<int> table_mem((size_t)n_row * n_col + 2 * guard);
    int *table = table_mem.p + guard;
    Dev<int> count_core(n_row), count_skin(n_row);
    {
        cudaTextureObject_t tex_aid = linear_tex(atm_id.p, sizeof(int) * nall, cudaCreateChannelDesc<int>());
        cudaTextureObject_t tex_coord = linear_tex(coord.p, sizeof(float4) * nall, cudaCreateChannelDesc<float4>());
        const int nslot = 32, nword = 5, threads = 128;
        const int shmem = (threads / WARPSZ) * (nslot * nword * (int)sizeof(int));
        const int blocks = std::max(1, std::min(148 * 16, (nbin + 3) / 4));
        GridConfig warp_cfg = make_int2(threads / WARPSZ, 1);
        const int n_part = warp_cfg.partition(nbin, (int)expected_bin_size, 0.0);
        gpu_build_neighbor_list<nslot, nword><<<blocks, threads, shmem>>>(
            tex_aid, tex_coord, count_core.p, count_skin.p, table, bin_loc.p, bin_size_local.p, stencil_len.p,
            stencil.p, stencil_pad, n_col, (r32)pow(cutneighmax - c.skin, 2.0), (r32)pow(cutneighmax, 2.0), nbin,
            std::max(n_part, 1));
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        std::vector<int> cc = count_core.down(n), cs = count_skin.down(n);
        for (int i = 0; i < n; ++i)
            if (cc[i] + cs[i] > n_col) fail("neighbour list overflow (raise rho_est)");
        gpu_join_neigh_list<<<(n + 127) / 128, 128>>>(count_core.p, count_skin.p, table, n_col, n);
        gpu_transpose_neigh_list<<<(n + 31) / 32, dim3(32, 8, 1)>>>(count_core.p, table, n_col, n);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        CK(cudaDestroyTextureObject(tex_aid));
        CK(cudaDestroyTextureObject(tex_coord));
    }
    std::vector<int> cnt = count_core.down(n);
    {
        std::vector<int> tab(table_mem.n);
        CK(cudaMemcpy(tab.data(), table_mem.p, tab.size() * sizeof(int), cudaMemcpyDeviceToHost));
        const int *T = tab.data() + guard;
        std::vector<int> rows;  // row i's entries in the reference's order, concatenated
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < cnt[i]; ++k) {
                const size_t a = (size_t)((i & ~31) + (k & 31)) * n_col + (k & ~31) + (i & 31);
                const int j = T[a];
                if (j < 0 || j >= nall) fail("list entry out of range");
                rows.push_back(j);
            }
        out.put("list_count", "i4", cnt.data(), n);
        out.put("list_rows", "i4", rows.data(), (int64_t)rows.size());
    }
    const int geo[6] = {mbin[0], mbin[1], mbin[2], n_col, n_bulk, ng};
    out.put("geometry_i", "i4", geo, 6);

    // ---- density pass: gpu_compute_rho (fix_aboundary_rho_meso.cu:119-165) ----
    cudaTextureObject_t tex_coord = linear_tex(coord.p, sizeof(float4) * nall, cudaCreateChannelDesc<float4>());
    cudaTextureObject_t tex_mass = linear_tex(amass.p, sizeof(double) * nall, cudaCreateChannelDesc<double>());
    const double rho_factor = 15.0 / (2.0 * M_PI * c.cut_rho * c.cut_rho * c.cut_rho * c.cut_rho * c.cut_rho);
    gpu_compute_rho<<<(n + 127) / 128, 128>>>(tex_coord, tex_mass, rho.p, amask.p, count_core.p, table, n_col, n,
                                              c.rho_bit, c.cut_rho, rho_factor);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    std::vector<double> rh = rho.down(nall);
    for (int g = 0; g < ng; ++g) rh[n + g] = rh[gsrc[g]];  // ghost rho by forward communication
    rho.up(rh.data(), nall);
    out.put("rho", "f8", rh.data(), n);

    // ---- wall volume fraction and bounce-back: gpu_aboundary (fix_aboundary_rho_meso.cu:220-287) ----
    Dev<double> phi(nall);
    if (c.arb_bc) {
        const double rc7 = pow(c.cut_phi, 7.0);
        const double phi_factor = 105.0 / (16.0 * M_PI * c.rho_wall * rc7);
        const double dw_factor = -315.0 / (4.0 * M_PI * c.rho_wall * rc7);
        const double dtf = 0.5 * c.dt, dtv = c.dt;  // FixArbitraryBoundaryRho::init, ftm2v = 1 (lj)
        Dev<double> bx(nall), by(nall), bz(nall), bvx(nall), bvy(nall), bvz(nall);
        CK(cudaMemcpy(bx.p, ax.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(by.p, ay.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(bz.p, az.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(bvx.p, avx.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(bvy.p, avy.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(bvz.p, avz.p, sizeof(double) * nall, cudaMemcpyDeviceToDevice));
        gpu_aboundary<<<(n + 127) / 128, 128>>>(amass.p, amask.p, bx.p, by.p, bz.p, bvx.p, bvy.p, bvz.p, phi.p,
                                                count_core.p, table, n_col, c.mobile_bit, c.wall_bit, n, c.cut_phi,
                                                phi_factor, dw_factor, c.phi_c, dtf, dtv);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        std::vector<double> ph = phi.down(n);
        out.put("phi", "f8", ph.data(), n);
        std::vector<double> b[6] = {bx.down(n), by.down(n), bz.down(n), bvx.down(n), bvy.down(n), bvz.down(n)};
        const char *nm[6] = {"bounce_x", "bounce_y", "bounce_z", "bounce_vx", "bounce_vy", "bounce_vz"};
        for (int q = 0; q < 6; ++q) out.put(nm[q], "f8", b[q].data(), n);
    }

    // ---- force pass: gpu_mdpd<1> (pair_mdpd_meso.cu:93-228) ----
    {
        cudaTextureObject_t tex_veloc = linear_tex(veloc.p, sizeof(float4) * nall, cudaCreateChannelDesc<float4>());
        cudaTextureObject_t tex_rho = linear_tex(rho.p, sizeof(double) * nall, cudaCreateChannelDesc<double>());
        cudaTextureObject_t tex_phi = linear_tex(phi.p, sizeof(double) * nall, cudaCreateChannelDesc<double>());
        Dev<double> fx(n), fy(n), fz(n), vxx(n), vyy(n), vzz(n), vxy(n), vxz(n), vyz(n), epair(n), coeffs(c.coeff.size());
        coeffs.up(c.coeff.data(), c.coeff.size());
        const int shmem = c.ntype * c.ntype * 6 * (int)sizeof(double);
        gpu_mdpd<1><<<(n + 127) / 128, 128, shmem>>>(tex_coord, tex_veloc, tex_rho, tex_phi, amask.p, fx.p, fy.p, fz.p,
                                                     vxx.p, vyy.p, vzz.p, vxy.p, vxz.p, vyz.p, count_core.p, table,
                                                     epair.p, coeffs.p, 1.0 / sqrt(c.dt), n_col, c.ntype, 0, n,
                                                     c.arb_bc, c.mobile_bit, c.wall_bit);
        CK(cudaGetLastError());
        CK(cudaDeviceSynchronize());
        const char *fn[10] = {"force_x", "force_y", "force_z", "virial_xx", "virial_yy",
                              "virial_zz", "virial_xy", "virial_xz", "virial_yz", "e_pair"};
        Dev<double> *fa[10] = {&fx, &fy, &fz, &vxx, &vyy, &vzz, &vxy, &vxz, &vyz, &epair};
        for (int q = 0; q < 10; ++q) {
            std::vector<double> h = fa[q]->down(n);
            out.put(fn[q], "f8", h.data(), n);
        }
        CK(cudaDestroyTextureObject(tex_veloc));
        CK(cudaDestroyTextureObject(tex_rho));
        CK(cudaDestroyTextureObject(tex_phi));
    }
    CK(cudaDestroyTextureObject(tex_coord));
    CK(cudaDestroyTextureObject(tex_mass));
    printf("ref_harness: %s: n=%d ghosts=%d bins=%dx%dx%d n_col=%d n_bulk=%d\n", argv[1], n, ng, mbin[0], mbin[1],
           mbin[2], n_col, n_bulk);
    return 0;
}
