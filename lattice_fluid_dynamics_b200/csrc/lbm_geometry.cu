// Solid masks, Bouzidi q values and the compacted boundary-link list,
// computed on the device.
//
// The reference builds the int32 solid mask and a dense 19-float-per-cell
// q table on the host (simulation/src/lbm.c:346-614, 964-1223) and
// uploads both.  Here every mask/q rule runs as a kernel with the same
// single-precision operation sequence (the library is built with
// --fmad=false), producing a dense q table in the reference's layout
// q[i + 19*cell] only transiently; the solver keeps the compacted list
// (links sorted by (cell, dir)) plus one flag byte per cell.
#include <cub/cub.cuh>

#include "lbm_d3q19.cuh"
#include "lbm_internal.h"

namespace lbm {

using namespace exact;

namespace {

constexpr int TPB = 256;

inline unsigned blocks_for(long long n) { return (unsigned)((n + TPB - 1) / TPB); }

__device__ __forceinline__ void cell_xyz(long long cell, int nx, int ny, int &x, int &y, int &z) {
    x = (int)(cell % nx);
    const long long r = cell / nx;
    y = (int)(r % ny);
    z = (int)(r / ny);
}

__global__ void k_fill(float *q, long long n, float v) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) q[k] = v;
}

__global__ void k_links_to_dense(const int32_t *lcell, const int32_t *ldir, const float *lq,
                                 long long nl, float *qd) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nl) qd[19LL * lcell[k] + ldir[k]] = lq[k];
}

// lbm.c:353-394
__global__ void k_aabb_solid(int32_t *solid, long long n, int nx, int ny, int x0, int x1, int y0,
                             int y1, int z0, int z1) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    int x, y, z;
    cell_xyz(cell, nx, ny, x, y, z);
    solid[cell] = (x >= x0 && x <= x1 && y >= y0 && y <= y1 && z >= z0 && z <= z1) ? 1 : 0;
}

// lbm.c:446-461
__global__ void k_sphere_solid(int32_t *solid, long long n, int nx, int ny, float scaleX,
                               float scaleY, float scaleZ, float cx, float cy, float cz, float r) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    int gx, gy, gz;
    cell_xyz(cell, nx, ny, gx, gy, gz);
    const float wx = __fdiv_rn((float)gx + 0.5f, scaleX) - 4.0f;
    const float wy = __fdiv_rn((float)gy + 0.5f, scaleY) - 2.0f;
    const float wz = __fdiv_rn((float)gz + 0.5f, scaleZ) - 2.0f;
    const float dx = wx - cx, dy = wy - cy, dz = wz - cz;
    solid[cell] = (dx * dx + dy * dy + dz * dz <= r * r) ? 1 : 0;
}

struct TriBounds {
    float minY, maxY, minZ, maxZ, maxX;
};

// lbm.c:990-1007
__global__ void k_tri_bounds(const float *tris, int nt, TriBounds *tb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const float *tri = tris + 12LL * t;
    const float v0y = tri[1], v0z = tri[2], v0x = tri[0];
    const float v1y = tri[5], v1z = tri[6], v1x = tri[4];
    const float v2y = tri[9], v2z = tri[10], v2x = tri[8];
    TriBounds b;
    b.minY = fminf(v0y, fminf(v1y, v2y));
    b.maxY = fmaxf(v0y, fmaxf(v1y, v2y));
    b.minZ = fminf(v0z, fminf(v1z, v2z));
    b.maxZ = fmaxf(v0z, fmaxf(v1z, v2z));
    b.maxX = fmaxf(v0x, fmaxf(v1x, v2x));
    tb[t] = b;
}

// lbm.c:1017-1095: +x ray parity inside test
__global__ void k_mesh_solid(int32_t *solid, long long n, int nx, int ny, float scaleX,
                             float scaleY, float scaleZ, const float *__restrict__ tris,
                             const TriBounds *__restrict__ tb, int nt, float minX, float minY,
                             float minZ, float maxX, float maxY, float maxZ) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    int gx, gy, gz;
    cell_xyz(cell, nx, ny, gx, gy, gz);
    const float wx = __fdiv_rn((float)gx + 0.5f, scaleX) - 4.0f;
    const float wy = __fdiv_rn((float)gy + 0.5f, scaleY) - 2.0f;
    const float wz = __fdiv_rn((float)gz + 0.5f, scaleZ) - 2.0f;
    int inside = 0;
    if (!(wx < minX || wx > maxX || wy < minY || wy > maxY || wz < minZ || wz > maxZ)) {
        int intersections = 0;
        for (int t = 0; t < nt; t++) {
            const TriBounds b = tb[t];
            if (wy < b.minY || wy > b.maxY || wz < b.minZ || wz > b.maxZ || wx > b.maxX) continue;
            const float *tri = tris + 12LL * t;
            const float v0x = tri[0], v0y = tri[1], v0z = tri[2];
            const float v1x = tri[4], v1y = tri[5], v1z = tri[6];
            const float v2x = tri[8], v2y = tri[9], v2z = tri[10];
            const float e1x = v1x - v0x, e1y = v1y - v0y, e1z = v1z - v0z;
            const float e2x = v2x - v0x, e2y = v2y - v0y, e2z = v2z - v0z;
            const float hx = 0.0f, hy = -e2z, hz = e2y;
            const float a = e1x * hx + e1y * hy + e1z * hz;
            if (a > -0.00001f && a < 0.00001f) continue;
            const float f = __fdiv_rn(1.0f, a);
            const float sx = wx - v0x, sy = wy - v0y, sz = wz - v0z;
            const float u = f * (sx * hx + sy * hy + sz * hz);
            if (u < 0.0f || u > 1.0f) continue;
            const float qx = sy * e1z - sz * e1y;
            const float qy = sz * e1x - sx * e1z;
            const float qz = sx * e1y - sy * e1x;
            const float v = f * qx;
            if (v < 0.0f || u + v > 1.0f) continue;
            const float dist = f * (e2x * qx + e2y * qy + e2z * qz);
            if (dist > 0.00001f) intersections++;
        }
        inside = (intersections % 2 == 1);
    }
    solid[cell] = inside ? 1 : 0;
}

enum { Q_HALF = 0, Q_SPHERE = 1, Q_MESH = 2 };

struct BodyParams {
    int mode;
    float scaleX, scaleY, scaleZ;
    float cx, cy, cz, r;            // sphere
    const float *tris;              // mesh
    const TriBounds *tb;
    int nt;
};

// lbm.c:1142-1204 (mesh per-link nearest hit)
__device__ float mesh_link_q(const BodyParams &p, float wx, float wy, float wz, float dx,
                             float dy, float dz) {
    float bestT = 2.0f;
    for (int t = 0; t < p.nt; t++) {
        const TriBounds b = p.tb[t];
        if (wy < b.minY || wy > b.maxY || wz < b.minZ || wz > b.maxZ || wx > b.maxX) continue;
        const float *tri = p.tris + 12LL * t;
        const float v0x = tri[0], v0y = tri[1], v0z = tri[2];
        const float v1x = tri[4], v1y = tri[5], v1z = tri[6];
        const float v2x = tri[8], v2y = tri[9], v2z = tri[10];
        const float e1x = v1x - v0x, e1y = v1y - v0y, e1z = v1z - v0z;
        const float e2x = v2x - v0x, e2y = v2y - v0y, e2z = v2z - v0z;
        const float hx = dy * e2z - dz * e2y;
        const float hy = dz * e2x - dx * e2z;
        const float hz = dx * e2y - dy * e2x;
        const float a = e1x * hx + e1y * hy + e1z * hz;
        if (a > -1e-6f && a < 1e-6f) continue;
        const float f = __fdiv_rn(1.0f, a);
        const float sx = wx - v0x, sy = wy - v0y, sz = wz - v0z;
        const float u = f * (sx * hx + sy * hy + sz * hz);
        if (u < 0.0f || u > 1.0f) continue;
        const float qx = sy * e1z - sz * e1y;
        const float qy = sz * e1x - sx * e1z;
        const float qz = sx * e1y - sy * e1x;
        const float v = f * (dx * qx + dy * qy + dz * qz);
        if (v < 0.0f || u + v > 1.0f) continue;
        const float tHit = f * (e2x * qx + e2y * qy + e2z * qz);
        if (tHit > 0.0f && tHit < bestT) bestT = tHit;
    }
    return bestT;
}

// Links from fluid cells into body cells (solid == 1): lbm.c:409-429
// (q = 0.5), :481-528 (analytic sphere), :1113-1212 (mesh).  qd was reset
// to -1 before.
__global__ void k_body_links(const int32_t *__restrict__ solid, float *qd, long long n, int nx,
                             int ny, int nz, BodyParams p) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    if (solid[cell] == 1) return;
    int gx, gy, gz;
    cell_xyz(cell, nx, ny, gx, gy, gz);
    const float wx = __fdiv_rn((float)gx + 0.5f, p.scaleX) - 4.0f;
    const float wy = __fdiv_rn((float)gy + 0.5f, p.scaleY) - 2.0f;
    const float wz = __fdiv_rn((float)gz + 0.5f, p.scaleZ) - 2.0f;
    for (int i = 1; i < 19; i++) {
        const int ex = cx(i), ey = cy(i), ez = cz(i);
        const int mx = gx + ex, my = gy + ey, mz = gz + ez;
        if (mx < 0 || mx >= nx || my < 0 || my >= ny || mz < 0 || mz >= nz) continue;
        if (solid[(long long)mx + (long long)nx * ((long long)my + (long long)ny * mz)] != 1)
            continue;
        float q = 0.5f;
        if (p.mode == Q_SPHERE) {
            const float dx = __fdiv_rn((float)ex, p.scaleX);
            const float dy = __fdiv_rn((float)ey, p.scaleY);
            const float dz = __fdiv_rn((float)ez, p.scaleZ);
            const float ox = wx - p.cx, oy = wy - p.cy, oz = wz - p.cz;
            const float a = dx * dx + dy * dy + dz * dz;
            const float b = 2.0f * (ox * dx + oy * dy + oz * dz);
            const float c = ox * ox + oy * oy + oz * oz - p.r * p.r;
            const float disc = b * b - 4.0f * a * c;
            if (disc >= 0.0f) {
                const float t = __fdiv_rn(-b - __fsqrt_rn(disc), 2.0f * a);
                if (t > 0.0f && t <= 1.0f) q = t;
            }
            if (q < 0.01f) q = 0.01f;
            if (q > 0.99f) q = 0.99f;
        } else if (p.mode == Q_MESH) {
            const float dx = __fdiv_rn((float)ex, p.scaleX);
            const float dy = __fdiv_rn((float)ey, p.scaleY);
            const float dz = __fdiv_rn((float)ez, p.scaleZ);
            const float bestT = mesh_link_q(p, wx, wy, wz, dx, dy, dz);
            q = (bestT <= 1.0f) ? bestT : 0.5f;
            if (q < 0.01f) q = 0.01f;
            if (q > 0.99f) q = 0.99f;
        }
        qd[19 * cell + i] = q;
    }
}

// lbm.c:557-570
__global__ void k_ground_solid(int32_t *solid, long long n_below) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell < n_below && solid[cell] == 0) solid[cell] = 2;
}

// lbm.c:573-600 (one plane of cells at z = gzAbove)
__global__ void k_ground_links(const int32_t *solid, float *qd, int nx, int ny, int gzAbove) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)nx * ny) return;
    const int gx = (int)(k % nx), gy = (int)(k / nx);
    const long long ci = (long long)gx + (long long)nx * ((long long)gy + (long long)ny * gzAbove);
    if (solid[ci] != 0) return;
    for (int i = 1; i < 19; i++) {
        if (cz(i) != -1) continue;
        const int mz = gzAbove + cz(i);
        const int my = gy + cy(i), mx = gx + cx(i);
        if (mx < 0 || mx >= nx || my < 0 || my >= ny || mz < 0) continue;
        const long long ni = (long long)mx + (long long)nx * ((long long)my + (long long)ny * mz);
        if (solid[ni] != 0 && qd[19 * ci + i] < 0.0f) qd[19 * ci + i] = 0.5f;
    }
}

__global__ void k_link_counts(const float *__restrict__ qd, long long n, uint32_t *mask,
                              int *nlinks, int *isb) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    uint32_t m = 0;
    for (int i = 0; i < 19; i++)
        if (qd[19 * cell + i] >= 0.0f) m |= 1u << i;
    mask[cell] = m;
    nlinks[cell] = __popc(m);
    isb[cell] = m ? 1 : 0;
}

__global__ void k_link_scatter(const float *__restrict__ qd, const uint32_t *__restrict__ mask,
                               const int *__restrict__ loff, const int *__restrict__ boff,
                               long long n, LinkList L) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    const uint32_t m = mask[cell];
    if (!m) return;
    const int b = boff[cell];
    const int first = loff[cell];
    L.bcell[b] = (int32_t)cell;
    L.bmask[b] = m;
    L.bfirst[b] = first;
    int k = first;
    for (int i = 0; i < 19; i++) {
        if (m & (1u << i)) {
            L.lq[k] = qd[19 * cell + i];
            L.lcell[k] = (int32_t)cell;
            L.ldir[k] = i;
            k++;
        }
    }
}

__global__ void k_flags(const int32_t *__restrict__ solid, const uint32_t *__restrict__ mask,
                        const int *__restrict__ boff, long long n, uint8_t *flags, int32_t *slot) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    const bool b = mask[cell] != 0;
    flags[cell] = (uint8_t)((solid[cell] & FLAG_SOLID_MASK) | (b ? FLAG_BOUNDARY : 0));
    slot[cell] = b ? boff[cell] : -1;
}

// lbm.c:616-668: one thread per projection column
__global__ void k_projected_area(const int32_t *__restrict__ solid, int nx, int ny, int nz,
                                 int axis, int *count) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int found = 0;
    if (axis == 0) {
        if (k >= (long long)ny * nz) return;
        const int gy = (int)(k % ny), gz = (int)(k / ny);
        const long long base = (long long)nx * ((long long)gy + (long long)ny * gz);
        for (int gx = 0; gx < nx && !found; gx++) found = solid[base + gx] == 1;
    } else if (axis == 1) {
        if (k >= (long long)nx * nz) return;
        const int gx = (int)(k % nx), gz = (int)(k / nx);
        for (int gy = 0; gy < ny && !found; gy++)
            found = solid[gx + (long long)nx * ((long long)gy + (long long)ny * gz)] == 1;
    } else {
        if (k >= (long long)nx * ny) return;
        const int gx = (int)(k % nx), gy = (int)(k / nx);
        for (int gz = 0; gz < nz && !found; gz++)
            found = solid[gx + (long long)nx * ((long long)gy + (long long)ny * gz)] == 1;
    }
    if (found) atomicAdd(count, 1);
}

}  // namespace

cudaError_t geo_fill_q(float *qd, long long n19, cudaStream_t s) {
    k_fill<<<blocks_for(n19), TPB, 0, s>>>(qd, n19, -1.0f);
    return cudaGetLastError();
}

cudaError_t geo_links_to_dense(const GridImpl &g, float *qd, cudaStream_t s) {
    cudaError_t e = geo_fill_q(qd, 19LL * g.n, s);
    if (e != cudaSuccess) return e;
    if (g.links.nl > 0)
        k_links_to_dense<<<blocks_for(g.links.nl), TPB, 0, s>>>(g.links.lcell, g.links.ldir,
                                                                g.links.lq, g.links.nl, qd);
    return cudaGetLastError();
}

cudaError_t geo_aabb(GridImpl &g, float *qd, float minX, float minY, float minZ, float maxX,
                     float maxY, float maxZ, cudaStream_t s) {
    const float scaleX = g.nx / 8.0f, scaleY = g.ny / 4.0f, scaleZ = g.nz / 4.0f;
    int gMinX = (int)((minX + 4.0f) * scaleX);
    int gMaxX = (int)((maxX + 4.0f) * scaleX);
    int gMinY = (int)((minY + 2.0f) * scaleY);
    int gMaxY = (int)((maxY + 2.0f) * scaleY);
    int gMinZ = (int)((minZ + 2.0f) * scaleZ);
    int gMaxZ = (int)((maxZ + 2.0f) * scaleZ);
    if (gMinX < 0) gMinX = 0;
    if (gMaxX >= g.nx) gMaxX = g.nx - 1;
    if (gMinY < 0) gMinY = 0;
    if (gMaxY >= g.ny) gMaxY = g.ny - 1;
    if (gMinZ < 0) gMinZ = 0;
    if (gMaxZ >= g.nz) gMaxZ = g.nz - 1;
    k_aabb_solid<<<blocks_for(g.n), TPB, 0, s>>>(g.solid, g.n, g.nx, g.ny, gMinX, gMaxX, gMinY,
                                                 gMaxY, gMinZ, gMaxZ);
    cudaError_t e = geo_fill_q(qd, 19LL * g.n, s);
    if (e != cudaSuccess) return e;
    BodyParams p{};
    p.mode = Q_HALF;
    p.scaleX = scaleX;
    p.scaleY = scaleY;
    p.scaleZ = scaleZ;
    k_body_links<<<blocks_for(g.n), TPB, 0, s>>>(g.solid, qd, g.n, g.nx, g.ny, g.nz, p);
    return cudaGetLastError();
}

cudaError_t geo_sphere(GridImpl &g, float *qd, float cx_, float cy_, float cz_, float r,
                       bool halfway, cudaStream_t s) {
    const float scaleX = g.nx / 8.0f, scaleY = g.ny / 4.0f, scaleZ = g.nz / 4.0f;
    k_sphere_solid<<<blocks_for(g.n), TPB, 0, s>>>(g.solid, g.n, g.nx, g.ny, scaleX, scaleY,
                                                   scaleZ, cx_, cy_, cz_, r);
    cudaError_t e = geo_fill_q(qd, 19LL * g.n, s);
    if (e != cudaSuccess) return e;
    BodyParams p{};
    p.mode = halfway ? Q_HALF : Q_SPHERE;
    p.scaleX = scaleX;
    p.scaleY = scaleY;
    p.scaleZ = scaleZ;
    p.cx = cx_;
    p.cy = cy_;
    p.cz = cz_;
    p.r = r;
    k_body_links<<<blocks_for(g.n), TPB, 0, s>>>(g.solid, qd, g.n, g.nx, g.ny, g.nz, p);
    return cudaGetLastError();
}

cudaError_t geo_ground(GridImpl &g, float *qd, float worldZ, cudaStream_t s) {
    const float scaleZ = g.nz / 4.0f;
    int gzGround = (int)((worldZ + 2.0f) * scaleZ);
    if (gzGround < 0) gzGround = 0;
    if (gzGround >= g.nz) gzGround = g.nz - 1;
    const long long below = (long long)g.nx * g.ny * (gzGround + 1);
    k_ground_solid<<<blocks_for(below), TPB, 0, s>>>(g.solid, below);
    const int gzAbove = gzGround + 1;
    if (gzAbove < g.nz)
        k_ground_links<<<blocks_for((long long)g.nx * g.ny), TPB, 0, s>>>(g.solid, qd, g.nx, g.ny,
                                                                          gzAbove);
    return cudaGetLastError();
}

cudaError_t geo_mesh(GridImpl &g, float *qd, const float *tris_dev, int ntris,
                     const float bbox[6], cudaStream_t s) {
    const float scaleX = g.nx / 8.0f, scaleY = g.ny / 4.0f, scaleZ = g.nz / 4.0f;
    TriBounds *tb = nullptr;
    cudaError_t e = cudaMallocAsync(&tb, sizeof(TriBounds) * (size_t)(ntris > 0 ? ntris : 1), s);
    if (e != cudaSuccess) return e;
    if (ntris > 0) k_tri_bounds<<<(ntris + TPB - 1) / TPB, TPB, 0, s>>>(tris_dev, ntris, tb);
    k_mesh_solid<<<blocks_for(g.n), TPB, 0, s>>>(g.solid, g.n, g.nx, g.ny, scaleX, scaleY, scaleZ,
                                                 tris_dev, tb, ntris, bbox[0], bbox[1], bbox[2],
                                                 bbox[3], bbox[4], bbox[5]);
    e = geo_fill_q(qd, 19LL * g.n, s);
    if (e == cudaSuccess) {
        BodyParams p{};
        p.mode = Q_MESH;
        p.scaleX = scaleX;
        p.scaleY = scaleY;
        p.scaleZ = scaleZ;
        p.tris = tris_dev;
        p.tb = tb;
        p.nt = ntris;
        k_body_links<<<blocks_for(g.n), TPB, 0, s>>>(g.solid, qd, g.n, g.nx, g.ny, g.nz, p);
        e = cudaGetLastError();
    }
    cudaFreeAsync(tb, s);
    return e;
}

void geo_free_links(LinkList &l) {
    cudaFree(l.bcell);
    cudaFree(l.bmask);
    cudaFree(l.bfirst);
    cudaFree(l.lq);
    cudaFree(l.lcell);
    cudaFree(l.ldir);
    l = LinkList{};
}

cudaError_t geo_compact(GridImpl &g, const float *qd, cudaStream_t s) {
    const long long n = g.n;
    uint32_t *mask = nullptr;
    int *nlinks = nullptr, *isb = nullptr, *loff = nullptr, *boff = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0, tb2 = 0;
    cudaError_t e = cudaSuccess;
#define GC(call)                       \
    do {                               \
        e = (call);                    \
        if (e != cudaSuccess) goto out; \
    } while (0)
    {
        GC(cudaMalloc(&mask, sizeof(uint32_t) * n));
        GC(cudaMalloc(&nlinks, sizeof(int) * n));
        GC(cudaMalloc(&isb, sizeof(int) * n));
        GC(cudaMalloc(&loff, sizeof(int) * n));
        GC(cudaMalloc(&boff, sizeof(int) * n));
        k_link_counts<<<blocks_for(n), TPB, 0, s>>>(qd, n, mask, nlinks, isb);
        GC(cudaGetLastError());
        GC(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, nlinks, loff, (int)n, s));
        GC(cub::DeviceScan::ExclusiveSum(nullptr, tb2, isb, boff, (int)n, s));
        if (tb2 > tmp_bytes) tmp_bytes = tb2;
        GC(cudaMalloc(&tmp, tmp_bytes));
        GC(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, nlinks, loff, (int)n, s));
        GC(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, isb, boff, (int)n, s));
        int lastl = 0, lasto = 0, lastb = 0, lastbo = 0;
        GC(cudaMemcpyAsync(&lastl, nlinks + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        GC(cudaMemcpyAsync(&lasto, loff + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        GC(cudaMemcpyAsync(&lastb, isb + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        GC(cudaMemcpyAsync(&lastbo, boff + n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        GC(cudaStreamSynchronize(s));
        const long long nl = (long long)lasto + lastl;
        const int nb = lastbo + lastb;
        geo_free_links(g.links);
        LinkList L;
        L.nb = nb;
        L.nl = nl;
        GC(cudaMalloc(&L.bcell, sizeof(int32_t) * (nb > 0 ? nb : 1)));
        GC(cudaMalloc(&L.bmask, sizeof(uint32_t) * (nb > 0 ? nb : 1)));
        GC(cudaMalloc(&L.bfirst, sizeof(int32_t) * (nb + 1)));
        GC(cudaMalloc(&L.lq, sizeof(float) * (nl > 0 ? nl : 1)));
        GC(cudaMalloc(&L.lcell, sizeof(int32_t) * (nl > 0 ? nl : 1)));
        GC(cudaMalloc(&L.ldir, sizeof(int32_t) * (nl > 0 ? nl : 1)));
        const int32_t nl32 = (int32_t)nl;
        GC(cudaMemcpyAsync(L.bfirst + nb, &nl32, sizeof(int32_t), cudaMemcpyHostToDevice, s));
        k_link_scatter<<<blocks_for(n), TPB, 0, s>>>(qd, mask, loff, boff, n, L);
        GC(cudaGetLastError());
        k_flags<<<blocks_for(n), TPB, 0, s>>>(g.solid, mask, boff, n, g.flags, g.slot);
        GC(cudaGetLastError());
        GC(cudaStreamSynchronize(s));
        g.links = L;
    }
out:
#undef GC
    cudaFree(mask);
    cudaFree(nlinks);
    cudaFree(isb);
    cudaFree(loff);
    cudaFree(boff);
    cudaFree(tmp);
    return e;
}

cudaError_t geo_projected_area(const GridImpl &g, int axis, int *count_dev, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(count_dev, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    long long cols = axis == 0 ? (long long)g.ny * g.nz
                   : axis == 1 ? (long long)g.nx * g.nz
                               : (long long)g.nx * g.ny;
    k_projected_area<<<blocks_for(cols), TPB, 0, s>>>(g.solid, g.nx, g.ny, g.nz, axis, count_dev);
    return cudaGetLastError();
}

}  // namespace lbm
