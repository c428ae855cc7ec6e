// Trilinear particle advection through the solver's velocity field.
//
// Reference: simulation/shaders/particle_lbm.comp:46-89 (world -> grid
// mapping, clamp to [0, N-1], eight-corner trilinear `mix`) and :207-293
// (relax the particle velocity toward 2 x the sampled lattice velocity
// with rate 5 dt, Euler position update, life decay 0.01 dt, respawn on
// exit/expiry), collisionMode 0.  The shader's respawn position comes from
// fract(sin(idx * k)); here it comes from a 32-bit counter hash of
// (seed, idx, k) so host and device produce identical particles.
//
// One thread per particle; the velocity field (16 B per cell) is read
// through the read-only path and mostly hits L2 for the lattice sizes the
// solver runs.
#include "lbm_internal.h"

namespace lbm {

namespace {

__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
    // "lowbias32" integer mixer (C. Wellons, hash-prospector)
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__host__ __device__ __forceinline__ float uniform01(uint32_t seed, uint32_t idx, uint32_t k) {
    const uint32_t h = mix32(mix32(mix32(seed ^ 0x9e3779b9U) + idx) + k * 0x85ebca6bU);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float mixf(float a, float b, float t) {
    return a * (1.0f - t) + b * t;
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    return fminf(fmaxf(v, lo), hi);
}

__global__ void __launch_bounds__(256) k_particles(LBMParticle *__restrict__ ps, int n,
                                                    const float4 *__restrict__ vel, int nx, int ny,
                                                    int nz, float dt, uint32_t seed) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    LBMParticle p = ps[idx];

    float gp[3];
    gp[0] = __fdiv_rn(p.x + 4.0f, 8.0f) * (float)nx;
    gp[1] = __fdiv_rn(p.y + 2.0f, 4.0f) * (float)ny;
    gp[2] = __fdiv_rn(p.z + 2.0f, 4.0f) * (float)nz;
    gp[0] = clampf(gp[0], 0.0f, (float)nx - 1.0f);
    gp[1] = clampf(gp[1], 0.0f, (float)ny - 1.0f);
    gp[2] = clampf(gp[2], 0.0f, (float)nz - 1.0f);
    const int dims[3] = {nx, ny, nz};
    int i0[3], i1[3];
    float fr[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float fl = floorf(gp[a]);
        i0[a] = (int)fl;
        i1[a] = min(i0[a] + 1, dims[a] - 1);
        fr[a] = gp[a] - fl;
    }
    auto V = [&](int x, int y, int z) {
        return __ldg(vel + ((long long)x + (long long)y * nx + (long long)z * nx * ny));
    };
    const float4 v000 = V(i0[0], i0[1], i0[2]);
    const float4 v100 = V(i1[0], i0[1], i0[2]);
    const float4 v010 = V(i0[0], i1[1], i0[2]);
    const float4 v110 = V(i1[0], i1[1], i0[2]);
    const float4 v001 = V(i0[0], i0[1], i1[2]);
    const float4 v101 = V(i1[0], i0[1], i1[2]);
    const float4 v011 = V(i0[0], i1[1], i1[2]);
    const float4 v111 = V(i1[0], i1[1], i1[2]);
    float flow[3];
    const float c000[3] = {v000.x, v000.y, v000.z}, c100[3] = {v100.x, v100.y, v100.z};
    const float c010[3] = {v010.x, v010.y, v010.z}, c110[3] = {v110.x, v110.y, v110.z};
    const float c001[3] = {v001.x, v001.y, v001.z}, c101[3] = {v101.x, v101.y, v101.z};
    const float c011[3] = {v011.x, v011.y, v011.z}, c111[3] = {v111.x, v111.y, v111.z};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float v00 = mixf(c000[c], c100[c], fr[0]);
        const float v10 = mixf(c010[c], c110[c], fr[0]);
        const float v01 = mixf(c001[c], c101[c], fr[0]);
        const float v11 = mixf(c011[c], c111[c], fr[0]);
        const float v0 = mixf(v00, v10, fr[1]);
        const float v1 = mixf(v01, v11, fr[1]);
        flow[c] = mixf(v0, v1, fr[2]) * 2.0f;
    }
    const float relaxation = 5.0f * dt;
    p.vx = mixf(p.vx, flow[0], relaxation);
    p.vy = mixf(p.vy, flow[1], relaxation);
    p.vz = mixf(p.vz, flow[2], relaxation);
    p.x += p.vx * dt;
    p.y += p.vy * dt;
    p.z += p.vz * dt;
    p.life -= 0.01f * dt;
    if (p.life <= 0.0f || p.x > 4.0f || fabsf(p.y) > 2.0f || fabsf(p.z) > 2.0f) {
        p.x = -4.0f;
        p.y = (uniform01(seed, (uint32_t)idx, 2u) - 0.5f) * 3.0f;
        p.z = (uniform01(seed, (uint32_t)idx, 3u) - 0.5f) * 3.0f;
        p.vx = 0.5f + uniform01(seed, (uint32_t)idx, 4u) * 0.2f;
        p.vy = 0.0f;
        p.vz = 0.0f;
        p.life = 1.0f;
    }
    ps[idx] = p;
}

}  // namespace

cudaError_t launch_particles(LBMParticle *p, int n, const float4 *vel, int nx, int ny, int nz,
                             float dt, uint32_t seed, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_particles<<<(n + 255) / 256, 256, 0, s>>>(p, n, vel, nx, ny, nz, dt, seed);
    return cudaGetLastError();
}

void particles_seed_host(LBMParticle *p, int n, uint32_t seed) {
    for (int i = 0; i < n; i++) {
        p[i].x = -4.0f;
        p[i].y = uniform01(seed, (uint32_t)i, 0u) * 4.0f - 2.0f;
        p[i].z = uniform01(seed, (uint32_t)i, 1u) * 4.0f - 2.0f;
        p[i].pad = 0.0f;
        p[i].vx = 0.0f;
        p[i].vy = 0.0f;
        p[i].vz = 0.0f;
        p[i].life = 1.0f;
    }
}

}  // namespace lbm
