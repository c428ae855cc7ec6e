// Device check of the D3Q19 collision: evaluates every operator on a large
// set of random cell states -- one cell per thread (collide()) and two cells
// per thread (the paired step's collision) -- and writes the post-collision
// populations to a binary file, [12][n][19]: slots 0-5 the one-cell results,
// 6-11 the two-cell results.  tests/test_collide_native_gpu.py builds it
// twice -- with the within-cell paired FP32 code (default) and with
// -DLBM_NO_PAIRED (one scalar operation per rounding) -- and requires all
// outputs to be bit-identical across builds and slot k to equal slot 6 + k.
// It also records FADD2/FMUL2/FFMA2 against the scalar operations on edge
// inputs.
//
// usage: collide_check <out.bin> <n_states>
//        collide_check --math <state.bin> <fi.bin> <m.bin> <n> <out.bin>
// The second form evaluates, for n given states, the device's equilibrium
// (feq one direction at a time, and the step's equilibria() of all 19), MRT
// forward transform and MRT inverse transform, then the two-cell step's
// paired versions of the last three, and writes them as float32 [7][n][19]; tests/test_collide_native_gpu.py compares them with the
// reference's own C mirrors of that arithmetic (simulation/test/
// test_lbm.c:43-187) through tests/golden/ref_math.json.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../lattice_fluid_dynamics_b200/csrc/lbm_step.cuh"

using namespace lbm;
using namespace lbm::exact;

__host__ __device__ inline unsigned hash32(unsigned x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
__host__ __device__ inline float u01(unsigned s, unsigned k) {
    return (float)(hash32(hash32(s * 0x9e3779b9U + 0x1234567U) + k * 0x85ebca6bU) >> 8) *
           (1.0f / 16777216.0f);
}

// A random state: weights times random perturbations; every 64th state is
// far from equilibrium so that the stability guard resets it.  States whose
// index is 0 mod 8 sit on the inlet plane (x = 0), 1 mod 8 on the outlet
// plane (x = NX - 1 = 9), the others inside (x = 5).
__device__ void random_state(int id, float (&f)[19]) {
    const float rho = 0.8f + 0.4f * u01(id, 0);
    const float amp = id % 64 == 3 ? 40.0f : 0.3f;
    for (int i = 0; i < 19; i++)
        f[i] = rho * wgt<float>(i) * (1.0f + amp * (u01(id, 10 + i) - 0.5f));
}
__device__ int state_x(int id) { return id % 8 == 0 ? 0 : id % 8 == 1 ? 9 : 5; }

// one kernel per operator (as in the library); operators: 0 BGK, 1 REG,
// 2 MRT, 3 BGK+S, 4 REG+S, 5 MRT+S.  Guard-reset cells output feq(1, 0).
template <int OP, bool SMAG>
__global__ void k_collide(int n, float tau, float omega, float smag18, int slot, float *out) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    float f[19], fn[19];
    random_state(id, f);
    float r, a, b, c;
    const int kind = prepare_cell<float>(f, 0, state_x(id), 10, 0.05f, 0.0f, 0.0f, r, a, b, c);
    if (kind != 0) {
        for (int i = 0; i < 19; i++) fn[i] = wgt<float>(i);
    } else {
        collide<float, OP, SMAG>(f, fn, r, a, b, c, tau, omega, smag18);
    }
    for (int i = 0; i < 19; i++) out[((long long)slot * n + id) * 19 + i] = fn[i];
}

// The same states collided two at a time by the paired step's collision
// (lane x = state 2p, lane y = state 2p + 1; 2p = 0 mod 8 puts lane x on the
// inlet and lane y on the outlet plane, as state_x() does for the scalar
// kernel).
template <int OP, bool SMAG>
__global__ void k_collide_pair(int n, float tau, float omega, float smag18, int slot,
                               float2 nz, float *out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * p + 1 >= n) return;
    float fa[19], fb[19];
    random_state(2 * p, fa);
    random_state(2 * p + 1, fb);
    const bool edge = (2 * p) % 8 == 0;
    float2 fn[19];
    bool ra, rb;
    pair_collide_fluid<OP, SMAG>(fa, fb, edge, edge, 0.05f, 0.0f, 0.0f, tau, omega, smag18, nz,
                                 fn, ra, rb);
    for (int i = 0; i < 19; i++) {
        out[((long long)slot * n + 2 * p) * 19 + i] = fn[i].x;
        out[((long long)slot * n + 2 * p + 1) * 19 + i] = fn[i].y;
    }
}

// paired instructions against scalar ones on edge operands
__global__ void k_pairs(int n, unsigned *bad) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    unsigned bx = hash32(id * 3 + 1), by = hash32(id * 3 + 2), bz = hash32(id * 3 + 3);
    if (id % 4 == 1) bx &= 0x807fffffu;  // subnormal or zero
    if (id % 4 == 2) by &= 0x807fffffu;
    float x = __uint_as_float(bx), y = __uint_as_float(by), z = __uint_as_float(bz);
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) return;
    const float2 X = make_float2(x, y), Y = make_float2(y, z), Z = make_float2(z, x);
    const float2 a = __fadd2_rn(X, Y), m = __fmul2_rn(X, Y), f = __ffma2_rn(X, Y, Z);
    auto same = [](float p, float q) { return __float_as_uint(p) == __float_as_uint(q) || (p != p && q != q); };
    if (!same(a.x, __fadd_rn(x, y)) || !same(a.y, __fadd_rn(y, z))) atomicAdd(bad + 0, 1u);
    if (!same(m.x, __fmul_rn(x, y)) || !same(m.y, __fmul_rn(y, z))) atomicAdd(bad + 1, 1u);
    if (!same(f.x, __fmaf_rn(x, y, z)) || !same(f.y, __fmaf_rn(y, z, x))) atomicAdd(bad + 2, 1u);
    // the solver's paired helpers, with constant and variable operands
    const float2 c = pfma(p2(1.0f, -4.0f), X, pmul(p2(0.25f, 3.0f), psub(padd(Y, p2(1.0f, 1.0f)), Z)));
    const float ex = __fmaf_rn(1.0f, x, __fmul_rn(0.25f, __fsub_rn(__fadd_rn(y, 1.0f), z)));
    const float ey = __fmaf_rn(-4.0f, y, __fmul_rn(3.0f, __fsub_rn(__fadd_rn(z, 1.0f), x)));
    if (!same(c.x, ex) || !same(c.y, ey)) atomicAdd(bad + 3, 1u);
    // a paired product feeding a paired subtract, on operands where fusing
    // would change the rounding (counted, not required to be zero)
    const float w = 1.0f + 0.5f * u01(id, 99), d0 = u01(id, 98), d1 = u01(id, 97);
    const float2 F2 = p2(0.3f + d1, 0.7f - d0), D2 = p2(d0, d1);
    const float2 g = psub(F2, pmul(p2(w, w), D2));
    if (!same(g.x, __fsub_rn(F2.x, __fmul_rn(w, D2.x))) ||
        !same(g.y, __fsub_rn(F2.y, __fmul_rn(w, D2.y))))
        atomicAdd(bad + 4, 1u);
}

__global__ void k_math(int n, const float *state, const float *fi, const float *mi, float *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float rho = state[4 * k], ux = state[4 * k + 1], uy = state[4 * k + 2],
                uz = state[4 * k + 3];
    float a[19], b[19];
    const long long o = (long long)k * 19, plane = (long long)n * 19;
    for (int i = 0; i < 19; i++) out[o + i] = feq<float>(i, rho, ux, uy, uz);
    equilibria<float>(rho, ux, uy, uz, a);
    for (int i = 0; i < 19; i++) out[plane + o + i] = a[i];
    for (int i = 0; i < 19; i++) a[i] = fi[o + i];
    mrt_forward<float>(a, b);
    for (int i = 0; i < 19; i++) out[2 * plane + o + i] = b[i];
    for (int i = 0; i < 19; i++) a[i] = mi[o + i];
    mrt_inverse<float>(a, b);
    for (int i = 0; i < 19; i++) out[3 * plane + o + i] = b[i];
}

// the paired step's versions, two states per thread (lanes x, y = 2p, 2p + 1)
__global__ void k_math_pair(int n, const float *state, const float *fi, const float *mi,
                            float2 nz, float *out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * p + 1 >= n) return;
    const long long ka = 2 * (long long)p, kb = ka + 1, plane = (long long)n * 19;
    auto two = [&](const float *v, long long stride, int j) {
        return make_float2(v[ka * stride + j], v[kb * stride + j]);
    };
    const float2 rho = two(state, 4, 0), ux = two(state, 4, 1), uy = two(state, 4, 2),
                 uz = two(state, 4, 3);
    const float2 u2 = padd(padd(pmulz(ux, ux, nz), pmulz(uy, uy, nz)), pmulz(uz, uz, nz));
    float2 A[19], B[19];
    pequilibria(rho, ux, uy, uz, u2, nz, A);
    auto put = [&](int slot, const float2 (&v)[19]) {
        for (int i = 0; i < 19; i++) {
            out[slot * plane + ka * 19 + i] = v[i].x;
            out[slot * plane + kb * 19 + i] = v[i].y;
        }
    };
    put(4, A);
    for (int i = 0; i < 19; i++) A[i] = two(fi, 19, i);
    pmrt_forward(A, nz, B);
    put(5, B);
    for (int i = 0; i < 19; i++) A[i] = two(mi, 19, i);
    pmrt_inverse(A, nz, B);
    put(6, B);
}

static bool read_file(const char *path, std::vector<float> &v) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    const size_t got = fread(v.data(), sizeof(float), v.size(), f);
    fclose(f);
    return got == v.size();
}

static int math_mode(int argc, char **argv) {
    if (argc < 7) return 2;
    const int n = atoi(argv[5]);
    if (n <= 0 || n % 2) return 2;
    std::vector<float> st((size_t)4 * n), fi((size_t)19 * n), mi((size_t)19 * n);
    if (!read_file(argv[2], st) || !read_file(argv[3], fi) || !read_file(argv[4], mi)) return 8;
    float *d_st = nullptr, *d_fi = nullptr, *d_mi = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_st, st.size() * 4) != cudaSuccess ||
        cudaMalloc(&d_fi, fi.size() * 4) != cudaSuccess ||
        cudaMalloc(&d_mi, mi.size() * 4) != cudaSuccess ||
        cudaMalloc(&d_out, (size_t)7 * 19 * n * 4) != cudaSuccess)
        return 3;
    cudaMemcpy(d_st, st.data(), st.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_fi, fi.data(), fi.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(d_mi, mi.data(), mi.size() * 4, cudaMemcpyHostToDevice);
    k_math<<<(n + 127) / 128, 128>>>(n, d_st, d_fi, d_mi, d_out);
    k_math_pair<<<(n / 2 + 127) / 128, 128>>>(n, d_st, d_fi, d_mi, make_float2(-0.0f, -0.0f),
                                             d_out);
    std::vector<float> h((size_t)7 * 19 * n);
    if (cudaMemcpy(h.data(), d_out, h.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return 4;
    FILE *fo = fopen(argv[6], "wb");
    if (!fo) return 5;
    fwrite(h.data(), sizeof(float), h.size(), fo);
    fclose(fo);
    cudaFree(d_st);
    cudaFree(d_fi);
    cudaFree(d_mi);
    cudaFree(d_out);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 6;
}

int main(int argc, char **argv) {
    if (argc >= 2 && strcmp(argv[1], "--math") == 0) return math_mode(argc, argv);
    if (argc < 3) return 2;
    const int n = atoi(argv[2]);
    float *d = nullptr;
    if (n % 2) return 2;
    if (cudaMalloc(&d, sizeof(float) * 19 * 12 * (size_t)n) != cudaSuccess) return 3;
    const float tau = 0.56f, om = 1.0f / tau, s18 = 18.0f * (0.1f * 0.1f);
    const int g = (n + 127) / 128;
    k_collide<OP_BGK, false><<<g, 128>>>(n, tau, om, s18, 0, d);
    k_collide<OP_REG, false><<<g, 128>>>(n, tau, om, s18, 1, d);
    k_collide<OP_MRT, false><<<g, 128>>>(n, tau, om, s18, 2, d);
    k_collide<OP_BGK, true><<<g, 128>>>(n, tau, om, s18, 3, d);
    k_collide<OP_REG, true><<<g, 128>>>(n, tau, om, s18, 4, d);
    k_collide<OP_MRT, true><<<g, 128>>>(n, tau, om, s18, 5, d);
    const float2 nz = make_float2(-0.0f, -0.0f);
    const int gp = (n / 2 + 127) / 128;
    k_collide_pair<OP_BGK, false><<<gp, 128>>>(n, tau, om, s18, 6, nz, d);
    k_collide_pair<OP_REG, false><<<gp, 128>>>(n, tau, om, s18, 7, nz, d);
    k_collide_pair<OP_MRT, false><<<gp, 128>>>(n, tau, om, s18, 8, nz, d);
    k_collide_pair<OP_BGK, true><<<gp, 128>>>(n, tau, om, s18, 9, nz, d);
    k_collide_pair<OP_REG, true><<<gp, 128>>>(n, tau, om, s18, 10, nz, d);
    k_collide_pair<OP_MRT, true><<<gp, 128>>>(n, tau, om, s18, 11, nz, d);
    std::vector<float> h((size_t)19 * 12 * n);
    if (cudaMemcpy(h.data(), d, sizeof(float) * h.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return 4;
    FILE *fo = fopen(argv[1], "wb");
    if (!fo) return 5;
    fwrite(h.data(), sizeof(float), h.size(), fo);
    fclose(fo);
    unsigned *bad = nullptr;
    cudaMalloc(&bad, 20);
    cudaMemset(bad, 0, 20);
    const int np = 1 << 22;
    k_pairs<<<np / 256, 256>>>(np, bad);
    unsigned hb[5];
    cudaMemcpy(hb, bad, 20, cudaMemcpyDeviceToHost);
    printf("pairs fadd2=%u fmul2=%u ffma2=%u helpers=%u mismatches of %d; paired mul->sub "
           "contracted in %u\n", hb[0], hb[1], hb[2], hb[3], np, hb[4]);
    if (hb[0] || hb[1] || hb[2] || hb[3]) return 7;
    cudaFree(d);
    cudaFree(bad);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 6;
}
