/*
 * Pin harness for the oracle -- TEST INFRASTRUCTURE ONLY.
 *
 *   ref_pin host   <out.json>  TEA words from the reference's premix_TEA (host side)
 *   ref_pin device <out.json>  gaussian_TEA<4> from the reference's device code, plus
 *                              probes of how nvcc contracts the expression forms the
 *                              reference uses for the pair distance (neigh_build_meso.cu:86-89),
 *                              the bin coordinate (neighbor_meso.cu:413-415, atom_meso.cu:294-296)
 *                              and the sub-bin offset (atom_meso.cu:297-299).
 *
 * The reference header src/USER-MESO/math_meso.h is included unmodified from the reference
 * tree; see the Makefile for the build recipe.
 */
#include "math_meso.h"

#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

static void put_u32(FILE *f, const char *name, const std::vector<uint32_t> &a, bool last = false)
{
    fprintf(f, "  \"%s\": [", name);
    for (size_t i = 0; i < a.size(); ++i) fprintf(f, "%s%u", i ? "," : "", a[i]);
    fprintf(f, "]%s\n", last ? "" : ",");
}

static void put_u64(FILE *f, const char *name, const std::vector<uint64_t> &a, bool last = false)
{
    fprintf(f, "  \"%s\": [", name);
    for (size_t i = 0; i < a.size(); ++i) fprintf(f, "%s\"%016llx\"", i ? "," : "", (unsigned long long)a[i]);
    fprintf(f, "]%s\n", last ? "" : ",");
}

template <class T> static uint64_t bits(T v)
{
    uint64_t u = 0;
    memcpy(&u, &v, sizeof(T));
    return u;
}

static int host_mode(const char *path)
{
    const int n = 512;
    std::mt19937_64 g(20240917);
    std::vector<uint32_t> a(n), b(n), w16(n), w32(n), w64(n);
    for (int i = 0; i < n; ++i) {
        a[i] = (uint32_t)g();
        b[i] = (uint32_t)g();
        if (i < 8) a[i] = i, b[i] = 7 - i;
        w16[i] = premix_TEA<16>(a[i], b[i]);
        w32[i] = premix_TEA<32>(a[i], b[i]);
        w64[i] = premix_TEA<64>(a[i], b[i]);
    }
    FILE *f = fopen(path, "w");
    if (!f) return 1;
    fprintf(f, "{\n  \"source\": \"premix_TEA<N> host instantiation of src/USER-MESO/math_meso.h\",\n");
    put_u32(f, "v0", a);
    put_u32(f, "v1", b);
    put_u32(f, "tea16", w16);
    put_u32(f, "tea32", w32);
    put_u32(f, "tea64", w64, true);
    fprintf(f, "}\n");
    fclose(f);
    return 0;
}

__global__ void k_gauss(const uint32_t *u, const uint32_t *v, double *out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = gaussian_TEA<4>(u[i] > v[i], u[i], v[i]);
}

__global__ void k_dr2(const float *a, const float *b, float *out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float dx = a[3 * i] - b[3 * i];
    float dy = a[3 * i + 1] - b[3 * i + 1];
    float dz = a[3 * i + 2] - b[3 * i + 2];
    float dr2 = dx * dx + dy * dy + dz * dz;
    out[i] = dr2;
}

__global__ void k_bin(const double *x, double lo, double inv, double *out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (x[i] - lo) * inv + 1.0;
}

__global__ void k_sub(const double *x, const unsigned *b, double bs, double ci, double *out, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (x[i] - (b[i] - 1) * bs) * ci;
}

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            fprintf(stderr, "CUDA error %s at %d\n", cudaGetErrorString(e_), __LINE__);        \
            return 2;                                                                          \
        }                                                                                      \
    } while (0)

template <class T> static T *up(const std::vector<T> &h)
{
    T *d = nullptr;
    if (cudaMalloc(&d, sizeof(T) * h.size()) != cudaSuccess) return nullptr;
    cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return d;
}

template <class T> static void down(std::vector<T> &h, const T *d)
{
    cudaMemcpy(h.data(), d, sizeof(T) * h.size(), cudaMemcpyDeviceToHost);
}

static int device_mode(const char *path)
{
    const int n = 4096;
    std::mt19937_64 g(777);
    std::vector<uint32_t> u(n), v(n);
    for (int i = 0; i < n; ++i) {
        u[i] = (uint32_t)g();
        v[i] = (uint32_t)g();
    }
    u[0] = 0, v[0] = 0;
    u[1] = 0xFFFFFFFFu, v[1] = 0xFFFFFFFFu;
    u[2] = 1, v[2] = 0;
    std::uniform_real_distribution<float> uf(-40.f, 40.f), dd(-1.3f, 1.3f);
    std::vector<float> a(3 * n), b(3 * n), r2(n);
    for (int i = 0; i < 3 * n; ++i) {
        a[i] = uf(g);
        b[i] = a[i] + dd(g);
    }
    std::uniform_real_distribution<double> ux(-43.0, 43.0);
    std::vector<double> x(n), tb(n), ts(n);
    std::vector<unsigned> bb(n);
    const double lo = -43.55, inv = 1.0 / 1.3065, bs = 1.3065, ci = 16.0 / 1.3065;
    for (int i = 0; i < n; ++i) {
        x[i] = ux(g);
        bb[i] = (unsigned)((x[i] - lo) / bs) + 1u;
    }
    uint32_t *du = up(u), *dv = up(v);
    float *da = up(a), *db = up(b);
    double *dx = up(x);
    unsigned *dbb = up(bb);
    double *dg = nullptr, *dtb = nullptr, *dts = nullptr;
    float *dr = nullptr;
    if (!du || !dv || !da || !db || !dx || !dbb) return 2;
    CK(cudaMalloc(&dg, sizeof(double) * n));
    CK(cudaMalloc(&dtb, sizeof(double) * n));
    CK(cudaMalloc(&dts, sizeof(double) * n));
    CK(cudaMalloc(&dr, sizeof(float) * n));
    int nb = (n + 127) / 128;
    k_gauss<<<nb, 128>>>(du, dv, dg, n);
    k_dr2<<<nb, 128>>>(da, db, dr, n);
    k_bin<<<nb, 128>>>(dx, lo, inv, dtb, n);
    k_sub<<<nb, 128>>>(dx, dbb, bs, ci, dts, n);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    std::vector<double> gv(n);
    down(gv, dg);
    down(r2, dr);
    down(tb, dtb);
    down(ts, dts);
    std::vector<uint64_t> gbits(n), abits(3 * n), bbits(3 * n), rbits(n), xb(n), tbb(n), tsb(n);
    std::vector<uint32_t> bu(bb.begin(), bb.end());
    for (int i = 0; i < n; ++i) {
        gbits[i] = bits(gv[i]);
        rbits[i] = bits(r2[i]);
        xb[i] = bits(x[i]);
        tbb[i] = bits(tb[i]);
        tsb[i] = bits(ts[i]);
    }
    for (int i = 0; i < 3 * n; ++i) {
        abits[i] = bits(a[i]);
        bbits[i] = bits(b[i]);
    }
    FILE *f = fopen(path, "w");
    if (!f) return 1;
    fprintf(f, "{\n  \"source\": \"gaussian_TEA<4> device instantiation of src/USER-MESO/math_meso.h, compute_80 PTX run on the GPU; nvcc contraction probes\",\n");
    fprintf(f, "  \"lo\": \"%016llx\", \"inv\": \"%016llx\", \"bs\": \"%016llx\", \"ci\": \"%016llx\",\n",
            (unsigned long long)bits(lo), (unsigned long long)bits(inv), (unsigned long long)bits(bs),
            (unsigned long long)bits(ci));
    put_u32(f, "u", u);
    put_u32(f, "v", v);
    put_u64(f, "gauss", gbits);
    put_u64(f, "dr2_a", abits);
    put_u64(f, "dr2_b", bbits);
    put_u64(f, "dr2", rbits);
    put_u64(f, "x", xb);
    put_u32(f, "bin", bu);
    put_u64(f, "bin_expr", tbb);
    put_u64(f, "sub_expr", tsb, true);
    fprintf(f, "}\n");
    fclose(f);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s host|device out.json\n", argv[0]);
        return 1;
    }
    if (!strcmp(argv[1], "host")) return host_mode(argv[2]);
    if (!strcmp(argv[1], "device")) return device_mode(argv[2]);
    return 1;
}
