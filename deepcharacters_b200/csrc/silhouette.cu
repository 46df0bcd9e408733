// Camera projection, projected-mesh boundary and the multi-view silhouette
// distance-transform loss (CameraProjectionGpu, MultiViewSilhouetteLossGpu and
// their gradient ops).
//
// References: CustomTensorFlowCPPOperators/src/CustomGPUOperators/
//   CameraProjectionOperator/CameraProjectionGPUOp{,Grad}.cu,
//   MultiViewSilhouetteLossOperator/MultiViewSilhouetteLossGPUOp{,Grad}.cu,
//   Skeletool/Mesh/CUDABasedRasterization.cu:168-200 (boundary test).
//
// The reference's data -> model term scans every vertex for every boundary
// pixel of the distance image (MultiViewSilhouetteLossGPUOp.cu:195-212).
// Here the boundary vertices of each view are binned into a grid whose cell
// edge is the search radius (30 * crop scale px), so a pixel only scans the
// 3x3 cells around it; the candidate with the smallest distance and, among
// equal distances, the smallest vertex id is the reference's first-strictly-
// smaller winner.
#include <algorithm>
#include <mutex>
#include <vector>

#include "hc_common.cuh"
#include "hc_math.cuh"
#include "renderer.cuh"

namespace hc {
namespace {

__device__ __forceinline__ float3 cam_point(const float* e, float3 p) {
    const float4 h = make_float4(p.x, p.y, p.z, 1.f);
    return make_float3(dot(make_float4(e[0], e[1], e[2], e[3]), h), dot(make_float4(e[4], e[5], e[6], e[7]), h),
                       dot(make_float4(e[8], e[9], e[10], e[11]), h));
}

__device__ __forceinline__ float3 cam_vector(const float* e, float3 p) {
    const float4 h = make_float4(p.x, p.y, p.z, 0.f);
    return make_float3(dot(make_float4(e[0], e[1], e[2], e[3]), h), dot(make_float4(e[4], e[5], e[6], e[7]), h),
                       dot(make_float4(e[8], e[9], e[10], e[11]), h));
}

// projectPointFloat (CameraUtil.h:108-137 of the custom-op utilities)
__device__ __forceinline__ float2 project2(const float* k, float3 p) {
    const float3 d1 = p * make_float3(k[0], k[1], k[2]);
    const float3 d2 = p * make_float3(k[3], k[4], k[5]);
    const float3 d3 = p * make_float3(k[6], k[7], k[8]);
    float x = d1.x + d1.y + d1.z;
    float y = d2.x + d2.y + d2.z;
    float z = d3.x + d3.y + d3.z;
    if (z > 0.0000001f) {
        x /= z;
        y /= z;
    } else {
        z = 0.00001f;
        x /= z;
        y /= z;
    }
    return make_float2(x, y);
}

__global__ void k_project(int B, int C, int N, const float* __restrict__ pts, const float* __restrict__ vecs,
                          const float* __restrict__ extr, const float* __restrict__ intr, int is_point,
                          float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * C * N) return;
    const int p = (int)(i % N);
    const int c = (int)((i / N) % C);
    const int b = (int)(i / ((long long)N * C));
    const float* e = extr + ((long long)b * C + c) * 12;
    const float* k = intr + ((long long)b * C + c) * 9;
    const float3 P = ld3(pts + ((long long)b * N + p) * 3);
    float2 r;
    if (is_point) {
        r = project2(k, cam_point(e, P));
    } else {
        const float3 cp = cam_point(e, P);
        const float3 np = cp + cam_vector(e, ld3(vecs + ((long long)b * N + p) * 3));
        const float2 a = project2(k, cp), bb = project2(k, np);
        float2 dvec = make_float2(bb.x - a.x, bb.y - a.y);
        const float inv = rsqrtf(dvec.x * dvec.x + dvec.y * dvec.y);
        r = make_float2(dvec.x * inv, dvec.y * inv);
    }
    out[2 * i] = r.x;
    out[2 * i + 1] = r.y;
}

// d(image point)/d(world point), summed over the cameras
// (CameraProjectionGPUOpGrad.cu:12-79; the normals get a zero gradient, :83-98)
__global__ void k_project_grad(int B, int C, int N, const float* __restrict__ gimg, const float* __restrict__ pts,
                               const float* __restrict__ extr, const float* __restrict__ intr, int is_point,
                               float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * N) return;
    const int p = (int)(i % N), b = (int)(i / N);
    float3 g = make_float3(0.f, 0.f, 0.f);
    if (is_point) {
        const float3 P = ld3(pts + i * 3);
        for (int c = 0; c < C; ++c) {
            const float* e = extr + ((long long)b * C + c) * 12;
            const float* k = intr + ((long long)b * C + c) * 9;
            const float3 cs = cam_point(e, P);
            const float ax = k[0], ay = k[4], gm = k[1];
            const float a00 = ax / cs.z, a01 = gm / cs.z, a02 = (-ax * cs.x - gm * cs.y) / (cs.z * cs.z);
            const float a11 = ay / cs.z, a12 = (-ay * cs.y) / (cs.z * cs.z);
            const float2 gi = make_float2(gimg[(((long long)b * C + c) * N + p) * 2],
                                          gimg[(((long long)b * C + c) * N + p) * 2 + 1]);
            // rows of dI/dv * dE/dv
            const float3 r0 = make_float3(a00 * e[0] + a01 * e[4] + a02 * e[8], a00 * e[1] + a01 * e[5] + a02 * e[9],
                                          a00 * e[2] + a01 * e[6] + a02 * e[10]);
            const float3 r1 = make_float3(a11 * e[4] + a12 * e[8], a11 * e[5] + a12 * e[9], a11 * e[6] + a12 * e[10]);
            g += r0 * gi.x + r1 * gi.y;
        }
    }
    st3(out + i * 3, g);
}

// Boundary vertices of the projected mesh: a vertex is on the boundary of a
// view if a pixel of the 3x3 window around its (truncated) projection is not
// covered (Skeletool/Mesh/CUDABasedRasterization.cu:168-200).  Coverage is the
// renderer's face buffer.
__global__ void k_boundary(int B, int C, int N, int W, int H, const float* __restrict__ p2d,
                           const int* __restrict__ face, unsigned char* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * C * N) return;
    const long long view = i / N;
    const int u = (int)p2d[2 * i], v = (int)p2d[2 * i + 1];
    unsigned char r = 0;
    if (u - 1 >= 0 && u + 1 < W && v - 1 >= 0 && v + 1 < H) {
        const int* F = face + view * H * W;
        for (int c = u - 1; c <= u + 1; ++c)
            for (int rr = v - 1; rr <= v + 1; ++rr)
                if (F[(long long)rr * W + c] < 0) r = 1;
    }
    out[i] = r;
}

// 2-D coverage of the projected mesh, the ProjectedMeshBoundaryGpu op's own
// raster (Skeletool/Mesh/CUDABasedRasterization.cu:80-145): every pixel of a
// triangle's clamped bounding box whose centre has image-space barycentrics
// within [-0.001, 1.001] is marked covered.  The barycentric expressions keep
// the reference's operation order, so coverage is bit-identical.  The binned
// passes only ever write "covered", so their unordered stores need no
// atomics (the hinted set-up, a kernel before them, also writes "open").  Pixels
// outside a triangle's conservative footprint (widened by the -0.001
// tolerance and the test's rounding error, see Footprint) are never tested
// against it: they cannot pass the exact test.

struct CoverTri {
    float2 a, b, c;
    float d1, d2;
    int x0, x1, y0, y1;
};

__device__ __forceinline__ bool cover_test(const CoverTri& t, float pu, float pv) {
    const float2 a = t.a, b = t.b, c = t.c;
    const float e2 = ((a.y - b.y) * pu + (b.x - a.x) * pv + a.x * b.y - b.x * a.y) / t.d2;
    const float e1 = ((a.y - c.y) * pu + (c.x - a.x) * pv + a.x * c.y - c.x * a.y) / t.d1;
    const float e0 = 1.f - e2 - e1;
    return e0 >= -0.001f && e1 >= -0.001f && e2 >= -0.001f && e0 <= 1.001f && e1 <= 1.001f && e2 <= 1.001f;
}

__device__ __forceinline__ Footprint cover_footprint(const CoverTri& t, int W, int H) {
    const float M = fmaxf(fmaxf(fmaxf(fabsf(t.a.x), fabsf(t.a.y)), fmaxf(fabsf(t.b.x), fabsf(t.b.y))),
                          fmaxf(fmaxf(fabsf(t.c.x), fabsf(t.c.y)), (float)max(W, H)));
    return footprint(make_float3(t.a.x, t.a.y, 2.f), make_float3(t.b.x, t.b.y, 2.f), make_float3(t.c.x, t.c.y, 2.f),
                     0.0011f, 2e-6f * M * M);
}

// Binned coverage.  The reference's one-thread-per-triangle sweep costs the
// summed box area of all triangles (10^4-pixel boxes of long thin triangles
// on deformed meshes, with most lanes idle); the coverage of a pixel only
// needs the first triangle that covers it.  So, as for the renderer, triangles are binned into 8x8-pixel
// tiles (the tiles their footprint reaches), and one CTA per tile tests each
// pixel against the tile's triangles until one covers it.  Pairs beyond a
// tile's bin capacity are swept at once by the binning thread (coverage is an
// OR of triangles, so any order of writes gives the same image).
constexpr int kCovTile = 8;
constexpr int kCovCap = 256;
constexpr int kCovSmall = 9;  // tiles a thread bins on its own (a 3x3 box of tiles)

// Image layout of the views of one call.  Views are frame-major (view =
// frame * n_cam + camera) and every camera has its own image size: a view's
// pixels (coverage image, distance image, per-pixel outputs), 8x8 coverage
// tiles and boundary-grid cells start at frame * (P, T, G) + the camera's
// offset in the frame.  When every camera has the same size the layout has
// n_cam = 1 (each view is a "frame" of one camera), so any number of cameras
// works; mixed sizes take up to kMaxLayoutCams cameras.  Passed by value.
constexpr int kMaxLayoutCams = 32;
struct CamImg {
    int W, H;          // image size (the distance image's U, V)
    int tiles_x;       // 8x8 coverage tiles per row
    int gx, gy;        // boundary-grid cells (edge: the search radius)
    long long pix;     // first pixel in the frame
    long long tile;    // first coverage tile in the frame
    long long cell;    // first grid cell in the frame
};
struct ImgLayout {
    int n_cam;
    long long P, T, G;  // pixels, coverage tiles, grid cells of a frame
    FastDiv fd_T;       // division by T
    CamImg cam[kMaxLayoutCams];
};
struct ViewImg {       // one view's image in the call's buffers
    int W, H, tiles_x, gx, gy;
    long long pix, tile, cell;
};

__device__ __forceinline__ ViewImg view_img(const ImgLayout& L, int view) {
    const int b = L.n_cam == 1 ? view : view / L.n_cam, c = view - b * L.n_cam;
    const CamImg& k = L.cam[c];
    ViewImg v;
    v.W = k.W;
    v.H = k.H;
    v.tiles_x = k.tiles_x;
    v.gx = k.gx;
    v.gy = k.gy;
    v.pix = b * L.P + k.pix;
    v.tile = b * L.T + k.tile;
    v.cell = b * L.G + k.cell;
    return v;
}

// the view of a coverage tile of the call (< 2^31 tiles), and the tile's index in the view
__device__ __forceinline__ int view_of_tile(const ImgLayout& L, long long key, int& tile) {
    const unsigned b = L.fd_T.div((unsigned)key);
    const long long r = key - (long long)b * L.T;
    int c = 0;
    while (c + 1 < L.n_cam && L.cam[c + 1].tile <= r) ++c;
    tile = (int)(r - L.cam[c].tile);
    return (int)b * L.n_cam + c;
}

__device__ __forceinline__ void cover_tri(int view, int f, int N, int W, int H, const int* __restrict__ faces,
                                          const float2* __restrict__ p2d, CoverTri& t) {
    const float2* P = p2d + (long long)view * N;
    t.a = P[faces[3 * f]];
    t.b = P[faces[3 * f + 1]];
    t.c = P[faces[3 * f + 2]];
    const float2 a = t.a, b = t.b, c = t.c;
    t.x0 = (int)fmaxf(fminf(a.x, fminf(b.x, c.x)) - 0.5f, 0);
    t.y0 = (int)fmaxf(fminf(a.y, fminf(b.y, c.y)) - 0.5f, 0);
    t.x1 = (int)fminf(fmaxf(a.x, fmaxf(b.x, c.x)) + 0.5f, W - 1);
    t.y1 = (int)fminf(fmaxf(a.y, fmaxf(b.y, c.y)) + 0.5f, H - 1);
    t.d2 = (a.y - b.y) * c.x + (b.x - a.x) * c.y + a.x * b.y - b.x * a.y;
    t.d1 = (a.y - c.y) * b.x + (c.x - a.x) * b.y + a.x * c.y - c.x * a.y;
}

// What the coverage tile stages per (view, triangle), written once by the
// binning pass: the footprint, the exact test's operands and the pixel box.
struct CovTileTri {
    float4 e0;  // footprint a0, b0, c0, a1
    float4 e1;  // b1, c1, a2, b2
    float4 e2;  // c2, d1, d2, interior threshold
    float4 ab;  // a.x, a.y, b.x, b.y
    float2 c;
    int2 bb;  // pixel box: x0 | x1 << 16, y0 | y1 << 16
};

__device__ __forceinline__ CovTileTri cover_record(const CoverTri& t, const Footprint& fp) {
    CovTileTri e;
    e.e0 = make_float4(fp.a[0], fp.b[0], fp.c[0], fp.a[1]);
    e.e1 = make_float4(fp.b[1], fp.c[1], fp.a[2], fp.b[2]);
    // interior threshold: a pixel centre inside every edge by three margins
    // passes the exact test whatever its rounding (the error of
    // e0 = 1 - e1 - e2 adds those of e1 and e2); disabled footprints get an
    // unreachable threshold
    const float mmax = fmaxf(fp.m[0], fmaxf(fp.m[1], fp.m[2]));
    e.e2 = make_float4(fp.c[2], t.d1, t.d2, mmax > 0.f ? 4.f * mmax : 3.0e38f);
    e.ab = make_float4(t.a.x, t.a.y, t.b.x, t.b.y);
    e.c = t.c;
    e.bb = make_int2(t.x0 | (t.x1 << 16), t.y0 | (t.y1 << 16));
    return e;
}

__device__ __forceinline__ Footprint record_footprint(const CovTileTri& e) {
    Footprint fp;
    fp.a[0] = e.e0.x;
    fp.b[0] = e.e0.y;
    fp.c[0] = e.e0.z;
    fp.a[1] = e.e0.w;
    fp.b[1] = e.e1.x;
    fp.c[1] = e.e1.y;
    fp.a[2] = e.e1.z;
    fp.b[2] = e.e1.w;
    fp.c[2] = e.e2.x;
    return fp;
}

// the reference's test of one pixel centre (only pixels of the triangle's
// clamped box are tested: a centre just outside the box can pass the widened
// barycentric test), with the footprint cull and the interior shortcut first
__device__ __forceinline__ bool cover_record_test(const CovTileTri& e, int px, int py) {
    if (px < (e.bb.x & 0xffff) || px > (e.bb.x >> 16) || py < (e.bb.y & 0xffff) || py > (e.bb.y >> 16)) return false;
    const float pu = px + 0.5f, pv = py + 0.5f;
    const float f0 = e.e0.x * pu + e.e0.y * pv + e.e0.z, f1 = e.e0.w * pu + e.e1.x * pv + e.e1.y,
                f2 = e.e1.z * pu + e.e1.w * pv + e.e2.x;
    if (f0 < 0.f || f1 < 0.f || f2 < 0.f) return false;
    if (f0 >= e.e2.w && f1 >= e.e2.w && f2 >= e.e2.w) return true;  // clearly inside
    CoverTri t;
    t.a = make_float2(e.ab.x, e.ab.y);
    t.b = make_float2(e.ab.z, e.ab.w);
    t.c = e.c;
    t.d1 = e.e2.y;
    t.d2 = e.e2.z;
    return cover_test(t, pu, pv);
}

struct CovBins {
    int* count;        // [tiles of the call]
    int* bins;         // [tiles of the call * kCovCap]
    CovTileTri* rec;   // [V*F]
    unsigned char* cover;       // coverage image, the layout's pixels
    const unsigned char* need;  // [tiles of the call] tiles with a pixel still open (NULL: every tile)
    const int* need_sum;        // [tiles of the call] per view: inclusive 2-D prefix sums of need (NULL: none)
    int* tiles;                 // [tiles of the call]: the tiles that received an entry, in no order
    int* n_tiles;               // their number (cleared before the binning pass)
    int* items;                 // [V*F]: hinted binning, the (view * F + triangle) pairs left by the cull
    int* n_items;               // their number (cleared before the cull)
};

// a bin slot of tile `key`; the tile's first slot also lists the tile for the
// tile pass (tile keys of a call fit 31 bits)
__device__ __forceinline__ int cov_claim(const CovBins& cb, long long key) {
    const int slot = atomicAdd(cb.count + key, 1);
    if (slot == 0) cb.tiles[atomicAdd(cb.n_tiles, 1)] = (int)key;
    return slot;
}

// needed tiles of a view in the tile box [tx0, tx1] x [ty0, ty1] (inclusive),
// from the view's 2-D prefix sums S (row-major, tiles_x per row)
__device__ __forceinline__ int need_in_box(const int* S, int tiles_x, int tx0, int ty0, int tx1, int ty1) {
    const int a = S[ty1 * tiles_x + tx1];
    const int b = ty0 > 0 ? S[(ty0 - 1) * tiles_x + tx1] : 0;
    const int c = tx0 > 0 ? S[ty1 * tiles_x + tx0 - 1] : 0;
    const int d = ty0 > 0 && tx0 > 0 ? S[(ty0 - 1) * tiles_x + tx0 - 1] : 0;
    return a - b - c + d;
}

// the pixels of one tile that a triangle covers, written at once (a pair
// beyond the tile's bin capacity)
__device__ void cov_sweep(const CovBins& cb, const ViewImg& vi, int tile, const CovTileTri& e) {
    const int ty = tile / vi.tiles_x, tx = tile - ty * vi.tiles_x;
    unsigned char* img = cb.cover + vi.pix;
    for (int v = ty * kCovTile; v < min(ty * kCovTile + kCovTile, vi.H); ++v)
        for (int u = tx * kCovTile; u < min(tx * kCovTile + kCovTile, vi.W); ++u)
            if (cover_record_test(e, u, v)) img[(long long)v * vi.W + u] = 1;
}

// Boundary flags from a per-pixel face hint (a renderer face buffer of the
// same views).  The flag of a vertex reads coverage only in the 3x3 window
// around its projection, and a window pixel is covered when the reference's
// 2-D test passes for its hint face, which is checked here exactly.  A vertex
// whose window lies in the image with all nine pixels covered that way is not
// on the boundary.  Otherwise the window's pixels are written to the
// coverage image (covered 1, open 0), the tiles of its open pixels are marked
// as needing the binned passes, and the vertex is flagged kPending and
// resolved from the coverage image after them.
// Any hint gives the flags of the unhinted op; a good one only saves work.
// Pixels outside every pending window are never read again, so only pending
// windows are written (the binned passes may see stale values elsewhere,
// which decide nothing), and every value written here is the same from every
// window that holds the pixel.
constexpr unsigned char kPending = 2;

// (6 CTAs of 256 per SM: the kernel waits on dependent gathers, and more
// resident warps hide them better than the registers they cost)
__global__ void __launch_bounds__(256, 6) k_bnd_hint(long long n, int N, int F, const __grid_constant__ ImgLayout L,
                           const float2* __restrict__ p2d, const int* __restrict__ faces,
                           const int* __restrict__ hint, unsigned char* __restrict__ cover,
                           unsigned char* __restrict__ need, unsigned char* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int view = (int)(i / N);
    const ViewImg vi = view_img(L, view);
    const int W = vi.W, H = vi.H;
    const float2 q = p2d[i];
    const int u = (int)q.x, v = (int)q.y;
    unsigned char r = 0;
    if (u - 1 >= 0 && u + 1 < W && v - 1 >= 0 && v + 1 < H) {
        int last = -1;
        CoverTri t;
        unsigned open = 0;  // bit 3 j + k: window pixel (row j, column k) is open
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int rr = v - 1 + j, c = u - 1 + k;
                const int f = hint[vi.pix + (long long)rr * W + c];
                bool cov = false;
                if (f >= 0 && f < F) {
                    if (f != last) {  // neighbouring pixels mostly share their hint face
                        cover_tri(view, f, N, W, H, faces, p2d, t);
                        last = f;
                    }
                    cov = c >= t.x0 && c <= t.x1 && rr >= t.y0 && rr <= t.y1 && cover_test(t, c + 0.5f, rr + 0.5f);
                }
                open |= (cov ? 0u : 1u) << (3 * j + k);
            }
        if (open) {  // only a pending window's pixels are read again
            r = kPending;
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int rr = v - 1 + j, c = u - 1 + k;
                    const bool op = (open >> (3 * j + k)) & 1u;
                    cover[vi.pix + (long long)rr * W + c] = op ? 0 : 1;
                    if (op) need[vi.tile + (long long)(rr / kCovTile) * vi.tiles_x + c / kCovTile] = 1;
                }
        }
    }
    out[i] = r;
}

// Per view, the inclusive 2-D prefix sums of the needed-tile flags, so that
// the binning pass drops a triangle whose tile box holds no needed tile with
// four loads.  One CTA per view: a warp per row (shuffle prefix sums over 32
// tiles at a time, carried along the row), then a thread per column down the
// rows.
constexpr int kNeedSumThreads = 512;
__global__ void __launch_bounds__(kNeedSumThreads) k_need_sum(const __grid_constant__ ImgLayout L,
                                                              const unsigned char* __restrict__ need,
                                                              int* __restrict__ sum) {
    const ViewImg vi = view_img(L, blockIdx.x);
    const int tx = vi.tiles_x, ty = (vi.H + kCovTile - 1) / kCovTile;
    const unsigned char* nd = need + vi.tile;
    int* S = sum + vi.tile;
    const int lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    for (int y = threadIdx.x >> 5; y < ty; y += nwarp) {
        int carry = 0;
        for (int x0 = 0; x0 < tx; x0 += 32) {  // warp-uniform
            const int x = x0 + lane;
            int v = x < tx ? nd[y * tx + x] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += u;
            }
            if (x < tx) S[y * tx + x] = carry + v;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < tx; x += blockDim.x) {
        int acc = 0;
        for (int y = 0; y < ty; ++y) {
            acc += S[y * tx + x];
            S[y * tx + x] = acc;
        }
    }
}

// One thread per (view, triangle): its record, then its tiles.  Boxes of up
// to kCovSmall tiles are binned by their own thread, one counter atomic per
// entry; larger boxes are taken by the whole warp, a tile per lane, reading
// the record back from global memory.
// (all 32 lanes of the warp call it together: the big boxes are shared out
// with warp votes; `sat` culls boxes without a needed tile)
__device__ __forceinline__ void cov_bin_item(int view, int fi, bool live, int N, int F,
                                             const int* __restrict__ faces, const float2* __restrict__ p2d,
                                             const CovBins& cb, const ImgLayout& L, bool sat) {
    const unsigned lane = threadIdx.x & 31;
    const ViewImg vi = view_img(L, view);
    const long long i = (long long)view * F + fi;
    int f = 0;
    CoverTri t;
    t.x0 = 0;
    t.x1 = -1;
    t.y0 = 0;
    t.y1 = -1;
    Footprint fp;
    if (live) {
        f = fi;
        cover_tri(view, f, N, vi.W, vi.H, faces, p2d, t);
    }
    bool nonempty = live && t.x1 >= t.x0 && t.y1 >= t.y0;
    const int tx0 = t.x0 / kCovTile, ty0 = t.y0 / kCovTile;
    const int ntx = nonempty ? t.x1 / kCovTile - tx0 + 1 : 0;
    int nt = nonempty ? ntx * (t.y1 / kCovTile - ty0 + 1) : 0;
    if (sat && nt > 0 &&  // a box without a needed tile needs nothing
        need_in_box(cb.need_sum + vi.tile, vi.tiles_x, tx0, ty0, t.x1 / kCovTile, t.y1 / kCovTile) == 0) {
        nonempty = false;
        nt = 0;
    }
    if (nonempty) {
        fp = cover_footprint(t, vi.W, vi.H);
        cb.rec[i] = cover_record(t, fp);
    }
    const bool big = nt > kCovSmall;
    const int my_nt = big ? 0 : nt;
    int cx = 0, cy = 0;  // column / row of tile k in the box, stepped without a division
    for (int k = 0; k < my_nt; ++k) {  // each lane walks its own small box
        const int tx = tx0 + cx, ty = ty0 + cy;
        if (++cx == ntx) {
            cx = 0;
            ++cy;
        }
        if (nt > 1 && !footprint_overlaps(fp, max(tx * kCovTile, t.x0), min(tx * kCovTile + kCovTile - 1, t.x1),
                                          max(ty * kCovTile, t.y0), min(ty * kCovTile + kCovTile - 1, t.y1)))
            continue;
        const int tile = ty * vi.tiles_x + tx;
        if (cb.need && !cb.need[vi.tile + tile]) continue;
        const long long key = vi.tile + tile;
        const int slot = cov_claim(cb, key);
        if (slot < kCovCap)
            cb.bins[key * kCovCap + slot] = f;
        else
            cov_sweep(cb, vi, tile, cb.rec[i]);
    }
    __syncwarp();  // the records of big triangles are read back by the other lanes
    unsigned pending = __ballot_sync(0xffffffffu, big);
    while (pending) {
        const int src = __ffs(pending) - 1;
        pending &= pending - 1;
        const int qv = __shfl_sync(0xffffffffu, view, src), qf = __shfl_sync(0xffffffffu, f, src);
        const ViewImg qi = view_img(L, qv);
        const CovTileTri q = cb.rec[(long long)qv * F + qf];
        const Footprint qfp = record_footprint(q);
        const int qx0 = q.bb.x & 0xffff, qx1 = q.bb.x >> 16, qy0 = q.bb.y & 0xffff, qy1 = q.bb.y >> 16;
        const int qtx0 = qx0 / kCovTile, qty0 = qy0 / kCovTile, qntx = qx1 / kCovTile - qtx0 + 1;
        const int qnt = qntx * (qy1 / kCovTile - qty0 + 1);
        // lane's tile k = lane + 32 j at (row cr, column cc), stepped by 32
        // (floor(a / n) for a <= 32 from one reciprocal, as in the raster binning)
        const float rq = 1.f / (float)qntx;
        const int step_r = (int)(32.5f * rq), step_c = 32 - step_r * qntx;
        int cr = (int)(((float)lane + 0.5f) * rq), cc = (int)lane - cr * qntx;
        for (int k = lane; k < qnt; k += 32) {
            const int tx = qtx0 + cc, ty = qty0 + cr;
            cc += step_c;
            cr += step_r;
            if (cc >= qntx) {
                cc -= qntx;
                ++cr;
            }
            if (!footprint_overlaps(qfp, max(tx * kCovTile, qx0), min(tx * kCovTile + kCovTile - 1, qx1),
                                    max(ty * kCovTile, qy0), min(ty * kCovTile + kCovTile - 1, qy1)))
                continue;
            const int tile = ty * qi.tiles_x + tx;
            const long long key = qi.tile + tile;
            if (cb.need && !cb.need[key]) continue;
            const int slot = cov_claim(cb, key);
            if (slot < kCovCap)
                cb.bins[key * kCovCap + slot] = qf;
            else
                cov_sweep(cb, qi, tile, q);
        }
    }
}

// the unhinted binning: every (view, triangle), grid (triangle blocks, views)
__global__ void __launch_bounds__(256, 4) k_cov_bin(int N, int F, const int* __restrict__ faces,
                                                    const float2* __restrict__ p2d, CovBins cb,
                                                    const __grid_constant__ ImgLayout L) {
    const int fi = blockIdx.x * blockDim.x + threadIdx.x;
    cov_bin_item(blockIdx.y, fi, fi < F, N, F, faces, p2d, cb, L, false);
}

// The hinted binning's first pass, light enough for full occupancy: the
// (view, triangle) pairs whose tile box holds a needed tile (most hold none),
// listed with one atomic per warp for k_cov_bin_list.
__global__ void k_cov_cull(int N, int F, const int* __restrict__ faces, const float2* __restrict__ p2d,
                           CovBins cb, const __grid_constant__ ImgLayout L) {
    const int fi = blockIdx.x * blockDim.x + threadIdx.x;
    const int view = blockIdx.y;
    const ViewImg vi = view_img(L, view);
    bool keep = false;
    if (fi < F) {  // no early exit: the whole warp takes part in the vote
        CoverTri t;
        cover_tri(view, fi, N, vi.W, vi.H, faces, p2d, t);
        keep = t.x1 >= t.x0 && t.y1 >= t.y0 &&
               need_in_box(cb.need_sum + vi.tile, vi.tiles_x, t.x0 / kCovTile, t.y0 / kCovTile, t.x1 / kCovTile,
                           t.y1 / kCovTile) > 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (!m) return;  // warp-uniform
    const int lane = threadIdx.x & 31, first = __ffs(m) - 1;
    int base = 0;
    if (lane == first) base = atomicAdd(cb.n_items, __popc(m));
    base = __shfl_sync(0xffffffffu, base, first);
    if (keep) cb.items[base + __popc(m & ((1u << lane) - 1u))] = view * F + fi;
}

// the hinted binning proper over the listed pairs (persistent, whole warps)
__global__ void __launch_bounds__(256, 4) k_cov_bin_list(int N, int F, const int* __restrict__ faces,
                                                         const float2* __restrict__ p2d, CovBins cb,
                                                         const __grid_constant__ ImgLayout L) {
    const int n = *cb.n_items;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int base = 32 * gw; base < n; base += 32 * nw) {  // warp-uniform
        const int i = base + lane;
        const bool live = i < n;
        const int item = live ? cb.items[i] : 0;
        const int view = item / F;
        cov_bin_item(view, item - view * F, live, N, F, faces, p2d, cb, L, false);
    }
}

// Persistent CTAs over the tiles that received entries (the binning pass
// lists them), one thread per pixel of the current tile: a pixel stops at the
// first binned triangle that covers it, the tile at the chunk after which all
// its pixels are covered.
__global__ void __launch_bounds__(kCovTile* kCovTile) k_cov_tile(int F, long long n_keys, CovBins cb,
                                                                  const __grid_constant__ ImgLayout L) {
    __shared__ CovTileTri s_t[kCovTile * kCovTile];
    const int listed = *cb.n_tiles;
    for (int it = blockIdx.x; it < listed; it += gridDim.x) {
        const long long key = cb.tiles[it];
        const int n = min(cb.count[key], kCovCap);
        int tile;
        const int view = view_of_tile(L, key, tile);
        const ViewImg vi = view_img(L, view);
        const int ty = tile / vi.tiles_x, tx = tile - ty * vi.tiles_x;
        const int px = tx * kCovTile + (int)threadIdx.x % kCovTile, py = ty * kCovTile + (int)threadIdx.x / kCovTile;
        const bool valid = px < vi.W && py < vi.H;
        unsigned char* pix = cb.cover + vi.pix + (long long)py * vi.W + px;
        bool covered = !valid || *pix;
        const CovTileTri* R = cb.rec + (long long)view * F;
        // every chunk starts with a barrier (so does the next tile: the staged
        // records of this one are no longer read there)
        for (int base = 0; base < n; base += kCovTile * kCovTile) {
            const int m = min(kCovTile * kCovTile, n - base);
            if (__syncthreads_and(covered)) break;  // every pixel of the tile is covered: stop staging
            if ((int)threadIdx.x < m) s_t[threadIdx.x] = R[cb.bins[key * kCovCap + base + threadIdx.x]];
            __syncthreads();
            for (int j = 0; j < m && !covered; ++j) covered = cover_record_test(s_t[j], px, py);
        }
        if (valid && covered && !*pix) *pix = 1;
    }
}

// boundary test of k_boundary against the coverage image instead of a face
// buffer; after k_bnd_hint only its pending vertices are evaluated
__global__ void k_boundary_cover(int B, int C, int N, const __grid_constant__ ImgLayout L,
                                 const float* __restrict__ p2d, const unsigned char* __restrict__ cover,
                                 bool pending_only, unsigned char* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * C * N) return;
    if (pending_only && out[i] != kPending) return;
    const ViewImg vi = view_img(L, (int)(i / N));
    const int W = vi.W, H = vi.H;
    const int u = (int)p2d[2 * i], v = (int)p2d[2 * i + 1];
    unsigned char r = 0;
    if (u - 1 >= 0 && u + 1 < W && v - 1 >= 0 && v + 1 < H) {
        const unsigned char* img = cover + vi.pix;
        for (int c = u - 1; c <= u + 1; ++c)
            for (int rr = v - 1; rr <= v + 1; ++rr)
                if (!img[(long long)rr * W + c]) r = 1;
    }
    out[i] = r;
}

__device__ __forceinline__ float dt_decode(unsigned char x) {
    float v = (int)x;
    if (v >= 127) v = (v - 127) * 2;
    return v;
}

// model -> data term per (frame, view, vertex) (MultiViewSilhouetteLossGPUOp.cu:11-138)
__global__ void k_sil_points(int B, int C, int N, const __grid_constant__ ImgLayout L, const float* __restrict__ p2d,
                             const float* __restrict__ n2d, const unsigned char* __restrict__ isb,
                             const unsigned char* __restrict__ dt, const float* __restrict__ crops,
                             float* __restrict__ residual, float* __restrict__ dtgrad) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * C * N) return;
    const long long view = i / N;
    const ViewImg vi = view_img(L, (int)view);
    const int U = vi.W;
    const float* cr = crops + view * 7;
    const float2 border = make_float2(cr[0], cr[1]);
    const float scale = cr[2];
    const float2 cmin = make_float2(cr[3], cr[4]), cmax = make_float2(cr[5], cr[6]);
    const float pu = p2d[2 * i], pv = p2d[2 * i + 1];
    const bool in_view = pu - 2 > cmin.x && pu + 2 < cmax.x && pv - 2 > cmin.y && pv + 2 < cmax.y;
    if (!in_view) {
        dtgrad[2 * i] = 0.f;
        dtgrad[2 * i + 1] = 0.f;
        residual[i] = 0.f;
        return;
    }
    const float fx = (pu - cmin.x) / scale + border.x, fy = (pv - cmin.y) / scale + border.y;
    const int x = (int)fx, y = (int)fy;
    const unsigned char* D = dt + vi.pix;
    float val = dt_decode(D[(long long)y * U + x]);
    const float f00 = dt_decode(D[(long long)(y - 1) * U + (x - 1)]), f01 = dt_decode(D[(long long)(y - 1) * U + x]);
    const float f02 = dt_decode(D[(long long)(y - 1) * U + (x + 1)]), f10 = dt_decode(D[(long long)y * U + (x - 1)]);
    const float f12 = dt_decode(D[(long long)y * U + (x + 1)]), f20 = dt_decode(D[(long long)(y + 1) * U + (x - 1)]);
    const float f21 = dt_decode(D[(long long)(y + 1) * U + x]), f22 = dt_decode(D[(long long)(y + 1) * U + (x + 1)]);
    const float du = (1.f / 8.f) * ((-1.f) * f00 + (+1.f) * f02 + (-2.f) * f10 + (+2.f) * f12 + (-1.f) * f20 + (+1.f) * f22);
    const float dv = (1.f / 8.f) * ((-1.f) * f00 + (-2.f) * f01 + (-1.f) * f02 + (+1.f) * f20 + (+2.f) * f21 + (+1.f) * f22);
    float2 dn = make_float2(du, dv), dnu = make_float2(du, dv);
    const bool inside = (int)D[(long long)y * U + x] <= 127;
    const float nonvanishing = (float)(int)(dn.x != 0 || dn.y != 0);
    const float boundary = (float)(int)(isb[i] != 0);
    if (inside) dn = make_float2(-dn.x, -dn.y);
    const float dn_dot = dn.x * n2d[2 * i] + dn.y * n2d[2 * i + 1];
    if (!(dn_dot >= 0.f) && inside) dnu = make_float2(-dnu.x, -dnu.y);
    val *= boundary;
    val *= nonvanishing;
    dnu = make_float2(dnu.x * boundary * nonvanishing, dnu.y * boundary * nonvanishing);
    dtgrad[2 * i] = dnu.x * (1.f / (255.f));
    dtgrad[2 * i + 1] = dnu.y * (1.f / (255.f));
    residual[i] = val * (1.f / (255.f));
}

// grid of boundary vertices per view: cell edge = search radius 30 * scale;
// a view's cells start at its layout cell offset
struct SilGrid {
    int* count;       // [cells of the call]
    int* start;       // [cells of the call + 1] per view prefix
    int* cursor;      // [cells of the call]
    int* items;       // [views * N]
};

__device__ __forceinline__ bool grid_cell(const float* cr, int gx, int gy, float px, float py, int& cx, int& cy) {
    // image-space box of the distance image, extended by one radius
    const float scale = cr[2], R = 30.f * scale;
    const float x0 = (0.f - cr[0]) * scale + cr[3] - R, y0 = (0.f - cr[1]) * scale + cr[4] - R;
    const float fx = floorf((px - x0) / R), fy = floorf((py - y0) / R);
    if (!(fx >= 0.f && fy >= 0.f && fx < (float)gx && fy < (float)gy)) return false;
    cx = (int)fx;
    cy = (int)fy;
    return true;
}

__global__ void k_grid_count(int B, int C, int N, const __grid_constant__ ImgLayout L, SilGrid g,
                             const float* __restrict__ p2d, const unsigned char* __restrict__ isb,
                             const float* __restrict__ crops) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * C * N || !isb[i]) return;
    const long long view = i / N;
    const ViewImg vi = view_img(L, (int)view);
    int cx, cy;
    if (!grid_cell(crops + view * 7, vi.gx, vi.gy, p2d[2 * i], p2d[2 * i + 1], cx, cy)) return;
    atomicAdd(&g.count[vi.cell + cy * vi.gx + cx], 1);
}

// exclusive scan of the cell counts, one CTA per view
__global__ void k_grid_scan(SilGrid g, const __grid_constant__ ImgLayout L) {
    const ViewImg vi = view_img(L, blockIdx.x);
    const int cells = vi.gx * vi.gy;
    __shared__ int s_part[1024];
    const int* cnt = g.count + vi.cell;
    int* st = g.start + vi.cell;
    // each thread scans a contiguous chunk
    const int per = (cells + blockDim.x - 1) / blockDim.x;
    const int lo = threadIdx.x * per, hi = min(cells, lo + per);
    int sum = 0;
    for (int c = lo; c < hi; ++c) sum += cnt[c];
    s_part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
        const int v = threadIdx.x >= (unsigned)off ? s_part[threadIdx.x - off] : 0;
        __syncthreads();
        s_part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = s_part[threadIdx.x] - sum;
    for (int c = lo; c < hi; ++c) {
        st[c] = run;
        g.cursor[vi.cell + c] = run;
        run += cnt[c];
    }
}

__global__ void k_grid_fill(int B, int C, int N, const __grid_constant__ ImgLayout L, SilGrid g,
                            const float* __restrict__ p2d, const unsigned char* __restrict__ isb,
                            const float* __restrict__ crops) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * C * N || !isb[i]) return;
    const long long view = i / N;
    const ViewImg vi = view_img(L, (int)view);
    int cx, cy;
    if (!grid_cell(crops + view * 7, vi.gx, vi.gy, p2d[2 * i], p2d[2 * i + 1], cx, cy)) return;
    const int slot = atomicAdd(&g.cursor[vi.cell + cy * vi.gx + cx], 1);
    g.items[view * (long long)N + slot] = (int)(i % N);
}

// data -> model term per distance-image pixel (MultiViewSilhouetteLossGPUOp.cu:142-240)
// Data -> model term of one pixel (MultiViewSilhouetteLossGPUOp.cu:98-138):
// a boundary pixel (DT value 127 with at least 4 boundary pixels in its 5x5
// window) takes the nearest boundary vertex within 30 * scale px (the
// minimum (distance, id): the reference's first strictly smaller one).
__device__ __forceinline__ void sil_pixel(long long view, const ViewImg& vi, int p, int dval, int N,
                                          const SilGrid& g, const float* __restrict__ p2d,
                                          const unsigned char* __restrict__ D, const float* __restrict__ crops,
                                          float& r0, float& r1, float& cl) {
    const int U = vi.W, V = vi.H;
    r0 = 0.f;
    r1 = 0.f;
    cl = -1.f;
    if (dval != 127) return;
    const int vid = p / U, uid = p - vid * U;
    int nb = 0;
    for (int j = -2; j <= 2; ++j)
        for (int k = -2; k <= 2; ++k) {
            const int yy = vid + j, xx = uid + k;
            if (yy >= 0 && yy < V && xx >= 0 && xx < U && (int)D[(long long)yy * U + xx] == 127) ++nb;
        }
    if (nb < 4) return;
    const float* cr = crops + view * 7;
    const float scale = cr[2];
    const float2 imgpos = make_float2(((float)uid - cr[0]) * scale + cr[3], ((float)vid - cr[1]) * scale + cr[4]);
    float bestd = 30.f * scale;
    int best = -1;
    int cx, cy;
    if (grid_cell(cr, vi.gx, vi.gy, imgpos.x, imgpos.y, cx, cy)) {
        for (int yy = max(cy - 1, 0); yy <= min(cy + 1, vi.gy - 1); ++yy)
            for (int xx = max(cx - 1, 0); xx <= min(cx + 1, vi.gx - 1); ++xx) {
                const long long cell = vi.cell + yy * vi.gx + xx;
                const int s0 = g.start[cell];
                const int n = g.count[cell];
                for (int q = 0; q < n; ++q) {
                    const int v = g.items[view * (long long)N + s0 + q];
                    const float* pp = p2d + (view * (long long)N + v) * 2;
                    const float2 dlt = make_float2(pp[0] - imgpos.x, pp[1] - imgpos.y);
                    const float dist = sqrtf(dlt.x * dlt.x + dlt.y * dlt.y);
                    if (dist < bestd || (dist == bestd && best >= 0 && v < best)) {
                        bestd = dist;
                        best = v;
                    }
                }
            }
    }
    if (best >= 0) {
        const float* pp = p2d + (view * (long long)N + best) * 2;
        r0 = (pp[0] - imgpos.x) / (30.f * scale);
        r1 = (pp[1] - imgpos.y) / (30.f * scale);
        cl = (float)best;
    }
}

// sil_pixel for a boundary pixel p (DT value 127) evaluated by a whole warp
// (p uniform): lanes 0-24 test the 5x5 neighbourhood, and the lanes share the
// grid cells' vertices.  Each lane keeps the sequential rule over its
// vertices (accept dist < 30 * scale, then the smaller id on equal distance),
// so the lane results merge into the same lexicographic minimum of
// (distance, vertex) as the one-thread loop.
__device__ __forceinline__ void sil_pixel_warp(long long view, const ViewImg& vi, int p, int N, const SilGrid& g,
                                               const float* __restrict__ p2d, const unsigned char* __restrict__ D,
                                               const float* __restrict__ crops, int lane, float& r0, float& r1,
                                               float& cl) {
    const int U = vi.W, V = vi.H;
    r0 = 0.f;
    r1 = 0.f;
    cl = -1.f;
    const int vid = p / U, uid = p - vid * U;
    bool on = false;
    if (lane < 25) {
        const int yy = vid + lane / 5 - 2, xx = uid + lane % 5 - 2;
        on = yy >= 0 && yy < V && xx >= 0 && xx < U && (int)D[(long long)yy * U + xx] == 127;
    }
    if (__popc(__ballot_sync(0xffffffffu, on)) < 4) return;
    const float* cr = crops + view * 7;
    const float scale = cr[2];
    const float2 imgpos = make_float2(((float)uid - cr[0]) * scale + cr[3], ((float)vid - cr[1]) * scale + cr[4]);
    float bestd = 30.f * scale;
    int best = -1;
    int cx, cy;
    if (grid_cell(cr, vi.gx, vi.gy, imgpos.x, imgpos.y, cx, cy)) {
        // lanes 0-8 load the 3x3 cells' ranges at once; the cells' vertices
        // are then dealt to the lanes through an inclusive prefix of the
        // counts, so the loads do not chain from cell to cell
        int cs = 0, cn = 0;
        if (lane < 9) {
            const int yy = cy - 1 + lane / 3, xx = cx - 1 + lane % 3;
            if (yy >= 0 && yy < vi.gy && xx >= 0 && xx < vi.gx) {
                const long long cell = vi.cell + yy * vi.gx + xx;
                cs = g.start[cell];
                cn = g.count[cell];
            }
        }
        int pre = cn;
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o) pre += t;
        }
        const int total = __shfl_sync(0xffffffffu, pre, 8);  // the prefix is complete over lanes 0-15
        for (int base = 0; base < total; base += 32) {
            const int q = base + lane;
            int c = 0;  // the cell holding entry q: the cells whose inclusive prefix is <= q
#pragma unroll
            for (int cc = 0; cc < 9; ++cc) c += __shfl_sync(0xffffffffu, pre, cc) <= q ? 1 : 0;
            c = min(c, 8);
            const int c_pre = __shfl_sync(0xffffffffu, pre, c), c_n = __shfl_sync(0xffffffffu, cn, c);
            const int c_s = __shfl_sync(0xffffffffu, cs, c);
            if (q < total) {
                const int v = g.items[view * (long long)N + c_s + (q - (c_pre - c_n))];
                const float* pp = p2d + (view * (long long)N + v) * 2;
                const float2 dlt = make_float2(pp[0] - imgpos.x, pp[1] - imgpos.y);
                const float dist = sqrtf(dlt.x * dlt.x + dlt.y * dlt.y);
                if (dist < bestd || (dist == bestd && best >= 0 && v < best)) {
                    bestd = dist;
                    best = v;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float od = __shfl_xor_sync(0xffffffffu, bestd, o);
        const int ob = __shfl_xor_sync(0xffffffffu, best, o);
        if (ob >= 0 && (best < 0 || od < bestd || (od == bestd && ob < best))) {
            bestd = od;
            best = ob;
        }
    }
    if (best >= 0) {
        const float* pp = p2d + (view * (long long)N + best) * 2;
        r0 = (pp[0] - imgpos.x) / (30.f * scale);
        r1 = (pp[1] - imgpos.y) / (30.f * scale);
        cl = (float)best;
    }
}

// Four consecutive pixels per thread, grid (pixel blocks of one view, views):
// one 4-byte DT load and 16-byte stores when the buffers allow (vec), and
// 32-bit index arithmetic.  Most pixels are not on the boundary and only
// write their zero outputs; in the vec path each boundary pixel is searched
// by a whole warp (sil_pixel_warp), the block's boundary pixels dealt to its
// warps in turn, instead of leaving one lane to search while the others wait.
// Launched with 256 threads (the shared lists hold the block's 1024 pixels).
__global__ void __launch_bounds__(256, 5) k_sil_pixels(int N, const __grid_constant__ ImgLayout L, SilGrid g,
                             const float* __restrict__ p2d, const unsigned char* __restrict__ dt,
                             const float* __restrict__ crops, float* __restrict__ residual1,
                             float* __restrict__ closest, int vec, double* __restrict__ sumsq1) {
    const long long view = blockIdx.y;
    const ViewImg vi = view_img(L, (int)view);
    const int P = vi.W * vi.H;
    const int p0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (4 * (int)(blockIdx.x * blockDim.x) >= P) return;  // blocks past a smaller view's pixels (CTA-uniform)
    const unsigned char* D = dt + vi.pix;
    const long long i0 = vi.pix + p0;
    if (vec) {  // P % 4 == 0 and aligned buffers: all four pixels of an active thread exist
        // The block's boundary pixels are listed in shared memory and dealt to
        // its warps in turn (a contour running along a row can put dozens in
        // one warp's 128 pixels); their results come back through shared
        // memory to the threads that own the pixels and store them.
        __shared__ int s_n;
        __shared__ unsigned short s_list[4 * 256];
        __shared__ float2 s_r[4 * 256];
        __shared__ float s_c[4 * 256];
        const bool active = p0 < P;  // no early exit: every thread takes part in the barriers
        int dv[4] = {0, 0, 0, 0};
        if (active) {
            const uchar4 d4 = *reinterpret_cast<const uchar4*>(D + p0);
            dv[0] = d4.x;
            dv[1] = d4.y;
            dv[2] = d4.z;
            dv[3] = d4.w;
        }
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (dv[k] == 127) s_list[atomicAdd(&s_n, 1)] = (unsigned short)(4 * threadIdx.x + k);
        __syncthreads();
        const int n = s_n, lane = threadIdx.x & 31;
        const int pb = 4 * (int)(blockIdx.x * blockDim.x);  // the block's first pixel
        for (int e = threadIdx.x >> 5; e < n; e += blockDim.x >> 5) {  // warp-uniform
            const int lp = s_list[e];
            float a0, a1, cl;
            sil_pixel_warp(view, vi, pb + lp, N, g, p2d, D, crops, lane, a0, a1, cl);
            if (lane == 0) {
                s_r[lp] = make_float2(a0, a1);
                s_c[lp] = cl;
            }
        }
        __syncthreads();
        float r[8], c[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            r[2 * k] = r[2 * k + 1] = 0.f;
            c[k] = -1.f;
            if (dv[k] == 127) {
                const float2 q = s_r[4 * threadIdx.x + k];
                r[2 * k] = q.x;
                r[2 * k + 1] = q.y;
                c[k] = s_c[4 * threadIdx.x + k];
            }
        }
        if (active) {
            reinterpret_cast<float4*>(residual1 + 2 * i0)[0] = make_float4(r[0], r[1], r[2], r[3]);
            reinterpret_cast<float4*>(residual1 + 2 * i0)[1] = make_float4(r[4], r[5], r[6], r[7]);
            *reinterpret_cast<float4*>(closest + i0) = make_float4(c[0], c[1], c[2], c[3]);
        }
        if (sumsq1) {  // launch-uniform: the squared residuals, one reduction per warp that has any
            float q = 0.f;
#pragma unroll
            for (int k = 0; k < 8; ++k) q += r[k] * r[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
            if (lane == 0 && q != 0.f) atomicAdd(sumsq1, (double)q);
        }
        return;
    }
    if (p0 >= P) return;
    float q = 0.f;
    for (int k = 0; k < 4 && p0 + k < P; ++k) {
        float r0, r1, cl;
        sil_pixel(view, vi, p0 + k, D[p0 + k], N, g, p2d, D, crops, r0, r1, cl);
        residual1[2 * (i0 + k)] = r0;
        residual1[2 * (i0 + k) + 1] = r1;
        closest[i0 + k] = cl;
        q += r0 * r0 + r1 * r1;
    }
    if (sumsq1 && q != 0.f) atomicAdd(sumsq1, (double)q);
}

// the squared-residual loss of the fused forward: weight x the accumulated sum
__global__ void k_sil_loss1(float weight, const double* __restrict__ sumsq1, float* __restrict__ loss) {
    *loss = (float)(weight * *sumsq1);
}

__global__ void k_sil_grad_points(long long n, const float* __restrict__ dtgrad, const float* __restrict__ g,
                                  float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[2 * i] = dtgrad[2 * i] * g[i];
    out[2 * i + 1] = dtgrad[2 * i + 1] * g[i];
}

// four pixels per thread on a (pixel block, view) grid: one 16-byte load of
// closest_vertex_id when the buffer allows (vec); the rare boundary pixels
// scatter their residual gradient to the closest vertex
__global__ void k_sil_grad_pixels(int N, const __grid_constant__ ImgLayout L, const float* __restrict__ g1,
                                  float s1, const float* __restrict__ closest, const float* __restrict__ crops,
                                  float* __restrict__ out, int vec) {
    const long long view = blockIdx.y;
    const ViewImg vi = view_img(L, (int)view);
    const int P = vi.W * vi.H;
    const int p0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (p0 >= P) return;
    const long long i0 = vi.pix + p0;
    float cl[4];
    if (vec) {
        const float4 c4 = *reinterpret_cast<const float4*>(closest + i0);
        cl[0] = c4.x;
        cl[1] = c4.y;
        cl[2] = c4.z;
        cl[3] = c4.w;
    } else {
        for (int k = 0; k < 4; ++k) cl[k] = p0 + k < P ? closest[i0 + k] : -1.f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int cv = (int)cl[k];
        if (cv < 0) continue;
        const float scale = crops[view * 7 + 2];
        float* o = out + (view * N + cv) * 2;
        atomicAdd(o, s1 * g1[2 * (i0 + k)] / (30.f * scale));  // (s1 x g) exact for s1 = 1
        atomicAdd(o + 1, s1 * g1[2 * (i0 + k) + 1] / (30.f * scale));
    }
}

}  // namespace
}  // namespace hc

using namespace hc;

extern "C" hc_status hc_camera_projection_forward(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                                  const float* points_global_space, const float* vectors_global_space,
                                                  const float* extrinsics, const float* intrinsics,
                                                  int32_t is_point, float* points_image_space) {
    clear_error();
    HC_REQUIRE(batch > 0 && n_cameras > 0 && n_points >= 0, "bad sizes");
    HC_REQUIRE(points_global_space && extrinsics && intrinsics && points_image_space, "NULL pointer");
    HC_REQUIRE(is_point || vectors_global_space, "vector mode needs vectors_global_space");
    const long long n = (long long)batch * n_cameras * n_points;
    if (n == 0) return HC_OK;
    k_project<<<div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(batch, n_cameras, n_points, points_global_space,
                                                                vectors_global_space, extrinsics, intrinsics,
                                                                is_point, points_image_space);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_camera_projection_backward(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                                   const float* points_image_space_grad,
                                                   const float* points_global_space, const float* extrinsics,
                                                   const float* intrinsics, int32_t is_point,
                                                   float* points_global_space_grad) {
    clear_error();
    HC_REQUIRE(batch > 0 && n_cameras > 0 && n_points >= 0, "bad sizes");
    HC_REQUIRE(points_image_space_grad && points_global_space && extrinsics && intrinsics && points_global_space_grad,
               "NULL pointer");
    const long long n = (long long)batch * n_points;
    if (n == 0) return HC_OK;
    k_project_grad<<<div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(batch, n_cameras, n_points,
                                                                     points_image_space_grad, points_global_space,
                                                                     extrinsics, intrinsics, is_point,
                                                                     points_global_space_grad);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_projected_mesh_boundary(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                                int32_t width, int32_t height, const float* points_image_space,
                                                const int32_t* face_buffer, uint8_t* is_boundary) {
    clear_error();
    HC_REQUIRE(batch > 0 && n_cameras > 0 && n_points >= 0 && width > 2 && height > 2, "bad sizes");
    HC_REQUIRE(points_image_space && face_buffer && is_boundary, "NULL pointer");
    const long long n = (long long)batch * n_cameras * n_points;
    if (n == 0) return HC_OK;
    k_boundary<<<div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(batch, n_cameras, n_points, width, height,
                                                                 points_image_space, face_buffer, is_boundary);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

namespace {

// The image layout of a call from its cameras' sizes (widths / heights [C],
// host arrays).  Cameras of one size give the one-camera layout.
hc_status make_layout(int32_t batch, int32_t n_cameras, const int32_t* widths, const int32_t* heights, ImgLayout& L,
                      long long& views) {
    HC_REQUIRE(batch > 0 && n_cameras > 0, "bad sizes");
    HC_REQUIRE(widths && heights, "NULL image sizes");
    bool uniform = true;
    for (int c = 0; c < n_cameras; ++c) {
        HC_REQUIRE(widths[c] > 2 && heights[c] > 2 && widths[c] < 32768 && heights[c] < 32768,
                   "bad image size %dx%d of camera %d", widths[c], heights[c], c);
        uniform = uniform && widths[c] == widths[0] && heights[c] == heights[0];
    }
    views = (long long)batch * n_cameras;
    HC_REQUIRE(views <= 65535, "too many views in one call (%lld)", views);
    const int nc = uniform ? 1 : n_cameras;
    HC_REQUIRE(nc <= kMaxLayoutCams, "at most %d cameras of different image sizes in one call (got %d)",
               kMaxLayoutCams, n_cameras);
    memset(&L, 0, sizeof(L));
    L.n_cam = nc;
    long long pix = 0, tile = 0, cell = 0;
    for (int c = 0; c < nc; ++c) {
        CamImg& k = L.cam[c];
        k.W = widths[c];
        k.H = heights[c];
        k.tiles_x = div_up(k.W, kCovTile);
        k.gx = div_up(k.W, 30) + 3;
        k.gy = div_up(k.H, 30) + 3;
        k.pix = pix;
        k.tile = tile;
        k.cell = cell;
        HC_REQUIRE((long long)k.W * k.H < (1ll << 31), "too many pixels in one view");
        pix += (long long)k.W * k.H;
        tile += (long long)k.tiles_x * div_up(k.H, kCovTile);
        cell += (long long)k.gx * k.gy;
    }
    L.P = pix;
    L.T = tile;
    L.G = cell;
    HC_REQUIRE(views / nc * L.T < (1ll << 31), "too many coverage tiles in one call");
    L.fd_T = FastDiv((unsigned)L.T);
    return HC_OK;
}

// widths / heights of n cameras of one size
struct SameSize {
    std::vector<int32_t> w, h;
    SameSize(int n, int32_t width, int32_t height) : w((size_t)std::max(n, 0), width), h((size_t)std::max(n, 0), height) {}
};

// the layout's largest view, in pixels (the per-pixel grids span it)
long long max_view_pixels(const ImgLayout& L) {
    long long m = 0;
    for (int c = 0; c < L.n_cam; ++c) m = std::max(m, (long long)L.cam[c].W * L.cam[c].H);
    return m;
}

// every view's pixel count a multiple of 4 (so every view starts 4-aligned)
// grid of a persistent kernel: as many CTAs as are resident at once (a
// second partial wave would run its strided work after everything else),
// never more than `items`
template <typename K>
unsigned resident_blocks(K kernel, int threads, long long items) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    return (unsigned)std::max<long long>(1, std::min<long long>(items, (long long)sms * per_sm));
}

bool pixels_by_four(const ImgLayout& L) {
    for (int c = 0; c < L.n_cam; ++c)
        if (((long long)L.cam[c].W * L.cam[c].H) % 4 != 0) return false;
    return true;
}

}  // namespace

struct hc_mesh_boundary_s {
    int F = 0, N = 0;
    DevBuf faces, p2d, cover, count, bins, rec, need, need_sum, tile_list, items;
};

extern "C" hc_status hc_mesh_boundary_create(hc_mesh_boundary* out, const int32_t* faces, int32_t n_faces,
                                             int32_t n_vertices) {
    clear_error();
    HC_REQUIRE(out && faces && n_faces > 0 && n_vertices > 0, "bad arguments");
    for (long long k = 0; k < 3LL * n_faces; ++k)
        HC_REQUIRE(faces[k] >= 0 && faces[k] < n_vertices, "face index %d out of range at %lld", faces[k], k);
    auto* h = new hc_mesh_boundary_s();
    h->F = n_faces;
    h->N = n_vertices;
    hc_status st = upload(h->faces, faces, 3 * (size_t)n_faces);
    if (st != HC_OK) {
        delete h;
        return st;
    }
    *out = h;
    return HC_OK;
}

extern "C" hc_status hc_mesh_boundary_destroy(hc_mesh_boundary h) {
    clear_error();
    if (!h) return HC_OK;
    h->faces.release();
    h->p2d.release();
    h->cover.release();
    h->count.release();
    h->bins.release();
    h->rec.release();
    h->need.release();
    h->need_sum.release();
    h->tile_list.release();
    h->items.release();
    delete h;
    return HC_OK;
}

static hc_status mesh_boundary_reserve_layout(hc_mesh_boundary h, long long views, const ImgLayout& L) {
    const size_t frames = (size_t)(views / L.n_cam);
    HC_TRY(h->p2d.ensure(sizeof(float) * 2 * (size_t)views * h->N));
    HC_TRY(h->cover.ensure(frames * (size_t)L.P));
    HC_TRY(h->count.ensure(sizeof(int) * frames * (size_t)L.T));
    HC_TRY(h->bins.ensure(sizeof(int) * frames * (size_t)L.T * kCovCap));
    HC_TRY(h->rec.ensure(sizeof(CovTileTri) * (size_t)views * h->F));
    HC_TRY(h->need.ensure(frames * (size_t)L.T));
    HC_TRY(h->need_sum.ensure(sizeof(int) * frames * (size_t)L.T));
    HC_TRY(h->tile_list.ensure(sizeof(int) * (frames * (size_t)L.T + 1)));
    HC_REQUIRE(views * h->F < (1ll << 31), "too many (view, triangle) pairs in one call");
    HC_TRY(h->items.ensure(sizeof(int) * ((size_t)views * h->F + 1)));
    return HC_OK;
}

extern "C" hc_status hc_mesh_boundary_reserve_sized(hc_mesh_boundary h, int32_t batch, int32_t n_cameras,
                                                    const int32_t* widths, const int32_t* heights) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    ImgLayout L;
    long long views = 0;
    HC_TRY(make_layout(batch, n_cameras, widths, heights, L, views));
    return mesh_boundary_reserve_layout(h, views, L);
}

extern "C" hc_status hc_mesh_boundary_reserve(hc_mesh_boundary h, int32_t batch, int32_t n_cameras, int32_t width,
                                              int32_t height) {
    const SameSize sz(n_cameras, width, height);
    return hc_mesh_boundary_reserve_sized(h, batch, n_cameras, sz.w.data(), sz.h.data());
}

static hc_status mesh_boundary_run(hc_mesh_boundary h, void* stream, int32_t batch, int32_t n_cameras,
                                   const int32_t* widths, const int32_t* heights, const float* points_global_space,
                                   const float* extrinsics, const float* intrinsics, const float* points_image_space,
                                   const int32_t* face_hint, uint8_t* is_boundary) {
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(is_boundary && (points_image_space || (points_global_space && extrinsics && intrinsics)),
               "NULL pointer");
    ImgLayout L;
    long long views = 0;
    HC_TRY(make_layout(batch, n_cameras, widths, heights, L, views));
    HC_TRY(mesh_boundary_reserve_layout(h, views, L));
    cudaStream_t s = (cudaStream_t)stream;
    const long long nv = views * h->N;
    const float* p2d = points_image_space;
    if (!p2d) {
        k_project<<<div_up(nv, 256), 256, 0, s>>>(batch, n_cameras, h->N, points_global_space, nullptr, extrinsics,
                                                  intrinsics, 1, h->p2d.as<float>());
        HC_CHECK_LAUNCH();
        p2d = h->p2d.as<float>();
    }
    const long long frames = views / L.n_cam;
    const long long n_keys = frames * L.T;  // coverage tiles of the call
    CovBins cb;
    cb.count = h->count.as<int>();
    cb.bins = h->bins.as<int>();
    cb.cover = h->cover.as<unsigned char>();
    cb.rec = h->rec.as<CovTileTri>();
    cb.need = nullptr;
    cb.need_sum = nullptr;
    cb.n_tiles = h->tile_list.as<int>();
    cb.tiles = cb.n_tiles + 1;
    cb.n_items = h->items.as<int>();
    cb.items = cb.n_items + 1;
    if (face_hint) {
        // final flags of the vertices whose window the hint covers; open
        // window pixels and their tiles for the binned passes
        HC_CUDA(cudaMemsetAsync(h->need.ptr, 0, (size_t)n_keys, s));
        k_bnd_hint<<<div_up(nv, 256), 256, 0, s>>>(nv, h->N, h->F, L, reinterpret_cast<const float2*>(p2d),
                                                   h->faces.as<int>(), face_hint, h->cover.as<unsigned char>(),
                                                   h->need.as<unsigned char>(), is_boundary);
        HC_CHECK_LAUNCH();
        k_need_sum<<<(unsigned)views, kNeedSumThreads, 0, s>>>(L, h->need.as<unsigned char>(), h->need_sum.as<int>());
        HC_CHECK_LAUNCH();
        cb.need = h->need.as<unsigned char>();
        cb.need_sum = h->need_sum.as<int>();
    } else {
        HC_CUDA(cudaMemsetAsync(h->cover.ptr, 0, (size_t)(frames * L.P), s));
    }
    HC_CUDA(cudaMemsetAsync(cb.count, 0, sizeof(int) * (size_t)n_keys, s));
    HC_CUDA(cudaMemsetAsync(cb.n_tiles, 0, sizeof(int), s));
    const float2* p2 = reinterpret_cast<const float2*>(p2d);
    if (face_hint) {  // cull, then bin the listed pairs
        HC_CUDA(cudaMemsetAsync(cb.n_items, 0, sizeof(int), s));
        k_cov_cull<<<dim3(div_up(h->F, 256), (unsigned)views), 256, 0, s>>>(h->N, h->F, h->faces.as<int>(), p2, cb, L);
        HC_CHECK_LAUNCH();
        k_cov_bin_list<<<resident_blocks(k_cov_bin_list, 256, views * h->F / 256 + 1), 256, 0, s>>>(
            h->N, h->F, h->faces.as<int>(), p2, cb, L);
    } else {
        k_cov_bin<<<dim3(div_up(h->F, 256), (unsigned)views), 256, 0, s>>>(h->N, h->F, h->faces.as<int>(), p2, cb, L);
    }
    HC_CHECK_LAUNCH();
    k_cov_tile<<<resident_blocks(k_cov_tile, kCovTile * kCovTile, n_keys), kCovTile * kCovTile, 0, s>>>(h->F, n_keys,
                                                                                                      cb, L);
    HC_CHECK_LAUNCH();
    k_boundary_cover<<<div_up(nv, 256), 256, 0, s>>>(batch, n_cameras, h->N, L, p2d, h->cover.as<unsigned char>(),
                                                     face_hint != nullptr, is_boundary);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

extern "C" hc_status hc_mesh_boundary_forward(hc_mesh_boundary h, void* stream, int32_t batch, int32_t n_cameras,
                                              int32_t width, int32_t height, const float* points_global_space,
                                              const float* extrinsics, const float* intrinsics,
                                              const float* points_image_space, uint8_t* is_boundary) {
    clear_error();
    const SameSize sz(n_cameras, width, height);
    return mesh_boundary_run(h, stream, batch, n_cameras, sz.w.data(), sz.h.data(), points_global_space, extrinsics,
                             intrinsics, points_image_space, nullptr, is_boundary);
}

extern "C" hc_status hc_mesh_boundary_forward_hinted(hc_mesh_boundary h, void* stream, int32_t batch,
                                                     int32_t n_cameras, int32_t width, int32_t height,
                                                     const float* points_global_space, const float* extrinsics,
                                                     const float* intrinsics, const float* points_image_space,
                                                     const int32_t* face_hint, uint8_t* is_boundary) {
    clear_error();
    HC_REQUIRE(face_hint, "face_hint is NULL");
    const SameSize sz(n_cameras, width, height);
    return mesh_boundary_run(h, stream, batch, n_cameras, sz.w.data(), sz.h.data(), points_global_space, extrinsics,
                             intrinsics, points_image_space, face_hint, is_boundary);
}

extern "C" hc_status hc_mesh_boundary_forward_sized(hc_mesh_boundary h, void* stream, int32_t batch,
                                                    int32_t n_cameras, const int32_t* widths, const int32_t* heights,
                                                    const float* points_global_space, const float* extrinsics,
                                                    const float* intrinsics, const float* points_image_space,
                                                    const int32_t* face_hint, uint8_t* is_boundary) {
    clear_error();
    return mesh_boundary_run(h, stream, batch, n_cameras, widths, heights, points_global_space, extrinsics,
                             intrinsics, points_image_space, face_hint, is_boundary);
}

struct hc_silhouette_s {
    DevBuf grid;
    size_t need = 0;
};

// grid scratch of a call: cell counts, starts (+1), cursors, and the boundary
// vertices of every view
static size_t grid_bytes(long long views, long long cells, int N) {
    return sizeof(int) * (size_t)(3 * cells + 1 + views * (long long)N);
}

extern "C" hc_status hc_silhouette_create(hc_silhouette* out) {
    clear_error();
    HC_REQUIRE(out, "out is NULL");
    *out = new hc_silhouette_s();
    return HC_OK;
}

extern "C" hc_status hc_silhouette_destroy(hc_silhouette h) {
    clear_error();
    if (!h) return HC_OK;
    h->grid.release();
    delete h;
    return HC_OK;
}

extern "C" hc_status hc_silhouette_reserve_sized(hc_silhouette h, int32_t batch, int32_t n_cameras, int32_t n_points,
                                                 const int32_t* widths, const int32_t* heights) {
    clear_error();
    HC_REQUIRE(h && n_points > 0, "bad sizes");
    ImgLayout L;
    long long views = 0;
    HC_TRY(make_layout(batch, n_cameras, widths, heights, L, views));
    HC_TRY(h->grid.ensure(grid_bytes(views, views / L.n_cam * L.G, n_points)));
    return HC_OK;
}

extern "C" hc_status hc_silhouette_reserve(hc_silhouette h, int32_t batch, int32_t n_cameras, int32_t n_points,
                                           int32_t resolution_u, int32_t resolution_v) {
    const SameSize sz(n_cameras, resolution_u, resolution_v);
    return hc_silhouette_reserve_sized(h, batch, n_cameras, n_points, sz.w.data(), sz.h.data());
}

namespace {

// Argument checks shared by the silhouette forward entry points; sets the
// layout and the grid scratch bytes the call needs.
hc_status sil_forward_plan(int32_t batch, int32_t n_cameras, int32_t n_points, const int32_t* widths,
                           const int32_t* heights, const float* points_image_space, const float* normals_image_space,
                           const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                           const float* multi_view_crops, const float* mv_dt_residual, const float* mv_dt_residual_1,
                           const float* dt_image_gradient, const float* closest_vertex_id, ImgLayout& L,
                           size_t& need) {
    HC_REQUIRE(batch > 0 && n_cameras > 0 && n_points > 0, "bad sizes");
    HC_REQUIRE(points_image_space && normals_image_space && is_boundary && distance_transform_image &&
                   multi_view_crops && mv_dt_residual && mv_dt_residual_1 && dt_image_gradient && closest_vertex_id,
               "NULL pointer");
    long long views = 0;
    HC_TRY(make_layout(batch, n_cameras, widths, heights, L, views));
    need = grid_bytes(views, views / L.n_cam * L.G, n_points);
    return HC_OK;
}

// The launches of one silhouette forward, the grid laid out in the scratch at
// `base` (at least the planned bytes).  The cell counts are cleared first:
// the scratch may hold a previous call's grid.
hc_status sil_forward_run(cudaStream_t s, int* base, const ImgLayout& L, int32_t batch, int32_t n_cameras,
                          int32_t n_points, const float* points_image_space, const float* normals_image_space,
                          const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                          const float* multi_view_crops, float* mv_dt_residual, float* mv_dt_residual_1,
                          float* dt_image_gradient, float* closest_vertex_id, float weight_1 = 0.f,
                          double* sumsq_1 = nullptr, float* loss_1 = nullptr) {
    const int N = n_points;
    const long long views = (long long)batch * n_cameras;
    const long long cells = views / L.n_cam * L.G;
    SilGrid g;
    g.count = base;
    g.start = base + cells;
    g.cursor = base + 2 * cells + 1;
    g.items = base + 3 * cells + 1;
    HC_CUDA(cudaMemsetAsync(g.count, 0, sizeof(int) * (size_t)cells, s));
    const long long np = views * N;
    k_sil_points<<<div_up(np, 256), 256, 0, s>>>(batch, n_cameras, N, L, points_image_space, normals_image_space,
                                                 is_boundary, distance_transform_image, multi_view_crops,
                                                 mv_dt_residual, dt_image_gradient);
    HC_CHECK_LAUNCH();
    k_grid_count<<<div_up(np, 256), 256, 0, s>>>(batch, n_cameras, N, L, g, points_image_space, is_boundary,
                                                 multi_view_crops);
    HC_CHECK_LAUNCH();
    k_grid_scan<<<(unsigned)views, 1024, 0, s>>>(g, L);
    HC_CHECK_LAUNCH();
    k_grid_fill<<<div_up(np, 256), 256, 0, s>>>(batch, n_cameras, N, L, g, points_image_space, is_boundary,
                                                multi_view_crops);
    HC_CHECK_LAUNCH();
    if (sumsq_1) HC_CUDA(cudaMemsetAsync(sumsq_1, 0, sizeof(double), s));
    {
        const int vec = pixels_by_four(L) && ((uintptr_t)distance_transform_image & 3) == 0 &&
                        ((uintptr_t)mv_dt_residual_1 & 15) == 0 && ((uintptr_t)closest_vertex_id & 15) == 0;
        k_sil_pixels<<<dim3(div_up(max_view_pixels(L), 4 * 256), (unsigned)views), 256, 0, s>>>(
            N, L, g, points_image_space, distance_transform_image, multi_view_crops, mv_dt_residual_1,
            closest_vertex_id, vec, sumsq_1);
    }
    HC_CHECK_LAUNCH();
    if (loss_1) {
        k_sil_loss1<<<1, 1, 0, s>>>(weight_1, sumsq_1, loss_1);
        HC_CHECK_LAUNCH();
    }
    return HC_OK;
}

hc_status sil_backward_run(cudaStream_t s, int32_t batch, int32_t n_cameras, int32_t n_points, const int32_t* widths,
                           const int32_t* heights, const float* mv_dt_grad, const float* mv_dt_grad_1,
                           const float* dt_image_grad, const float* closest_vertex_id, const float* multi_view_crops,
                           float* points_image_space_grad, float scale_1 = 1.f) {
    HC_REQUIRE(batch > 0 && n_cameras > 0 && n_points > 0, "bad sizes");
    HC_REQUIRE(mv_dt_grad && mv_dt_grad_1 && dt_image_grad && closest_vertex_id && multi_view_crops &&
                   points_image_space_grad,
               "NULL pointer");
    ImgLayout L;
    long long views = 0;
    HC_TRY(make_layout(batch, n_cameras, widths, heights, L, views));
    const long long np = views * n_points;
    k_sil_grad_points<<<div_up(np, 256), 256, 0, s>>>(np, dt_image_grad, mv_dt_grad, points_image_space_grad);
    HC_CHECK_LAUNCH();
    const int vec = pixels_by_four(L) && ((uintptr_t)closest_vertex_id & 15) == 0;
    k_sil_grad_pixels<<<dim3(div_up(max_view_pixels(L), 4 * 256), (unsigned)views), 256, 0, s>>>(
        n_points, L, mv_dt_grad_1, scale_1, closest_vertex_id, multi_view_crops, points_image_space_grad, vec);
    HC_CHECK_LAUNCH();
    return HC_OK;
}

}  // namespace

extern "C" hc_status hc_silhouette_forward_sized(hc_silhouette h, void* stream, int32_t batch, int32_t n_cameras,
                                                 int32_t n_points, const int32_t* widths, const int32_t* heights,
                                                 const float* points_image_space, const float* normals_image_space,
                                                 const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                                                 const float* multi_view_crops, float* mv_dt_residual,
                                                 float* mv_dt_residual_1, float* dt_image_gradient,
                                                 float* closest_vertex_id) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    ImgLayout L;
    size_t need = 0;
    HC_TRY(sil_forward_plan(batch, n_cameras, n_points, widths, heights, points_image_space, normals_image_space,
                            is_boundary, distance_transform_image, multi_view_crops, mv_dt_residual,
                            mv_dt_residual_1, dt_image_gradient, closest_vertex_id, L, need));
    HC_TRY(h->grid.ensure(need));
    return sil_forward_run((cudaStream_t)stream, h->grid.as<int>(), L, batch, n_cameras, n_points,
                           points_image_space, normals_image_space, is_boundary, distance_transform_image,
                           multi_view_crops, mv_dt_residual, mv_dt_residual_1, dt_image_gradient, closest_vertex_id);
}

extern "C" hc_status hc_silhouette_forward_sumsq_sized(
    hc_silhouette h, void* stream, int32_t batch, int32_t n_cameras, int32_t n_points, const int32_t* widths,
    const int32_t* heights, const float* points_image_space, const float* normals_image_space,
    const uint8_t* is_boundary, const uint8_t* distance_transform_image, const float* multi_view_crops,
    float* mv_dt_residual, float* mv_dt_residual_1, float* dt_image_gradient, float* closest_vertex_id,
    float weight_1, double* sumsq_1, float* loss_1) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(sumsq_1 && loss_1, "NULL pointer");
    ImgLayout L;
    size_t need = 0;
    HC_TRY(sil_forward_plan(batch, n_cameras, n_points, widths, heights, points_image_space, normals_image_space,
                            is_boundary, distance_transform_image, multi_view_crops, mv_dt_residual,
                            mv_dt_residual_1, dt_image_gradient, closest_vertex_id, L, need));
    HC_TRY(h->grid.ensure(need));
    return sil_forward_run((cudaStream_t)stream, h->grid.as<int>(), L, batch, n_cameras, n_points,
                           points_image_space, normals_image_space, is_boundary, distance_transform_image,
                           multi_view_crops, mv_dt_residual, mv_dt_residual_1, dt_image_gradient, closest_vertex_id,
                           weight_1, sumsq_1, loss_1);
}

extern "C" hc_status hc_silhouette_forward(hc_silhouette h, void* stream, int32_t batch, int32_t n_cameras,
                                           int32_t n_points, int32_t resolution_u, int32_t resolution_v,
                                           const float* points_image_space, const float* normals_image_space,
                                           const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                                           const float* multi_view_crops, float* mv_dt_residual,
                                           float* mv_dt_residual_1, float* dt_image_gradient,
                                           float* closest_vertex_id) {
    const SameSize sz(n_cameras, resolution_u, resolution_v);
    return hc_silhouette_forward_sized(h, stream, batch, n_cameras, n_points, sz.w.data(), sz.h.data(),
                                       points_image_space, normals_image_space, is_boundary,
                                       distance_transform_image, multi_view_crops, mv_dt_residual, mv_dt_residual_1,
                                       dt_image_gradient, closest_vertex_id);
}

extern "C" hc_status hc_silhouette_backward(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                            int32_t resolution_u, int32_t resolution_v, const float* mv_dt_grad,
                                            const float* mv_dt_grad_1, const float* dt_image_grad,
                                            const float* closest_vertex_id, const float* multi_view_crops,
                                            float* points_image_space_grad) {
    clear_error();
    const SameSize sz(n_cameras, resolution_u, resolution_v);
    return sil_backward_run((cudaStream_t)stream, batch, n_cameras, n_points, sz.w.data(), sz.h.data(), mv_dt_grad,
                            mv_dt_grad_1, dt_image_grad, closest_vertex_id, multi_view_crops,
                            points_image_space_grad);
}

extern "C" hc_status hc_silhouette_backward_sized(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                                  const int32_t* widths, const int32_t* heights,
                                                  const float* mv_dt_grad, const float* mv_dt_grad_1,
                                                  const float* dt_image_grad, const float* closest_vertex_id,
                                                  const float* multi_view_crops, float* points_image_space_grad) {
    clear_error();
    return sil_backward_run((cudaStream_t)stream, batch, n_cameras, n_points, widths, heights, mv_dt_grad,
                            mv_dt_grad_1, dt_image_grad, closest_vertex_id, multi_view_crops,
                            points_image_space_grad);
}

extern "C" hc_status hc_silhouette_backward_scaled_sized(void* stream, int32_t batch, int32_t n_cameras,
                                                         int32_t n_points, const int32_t* widths,
                                                         const int32_t* heights, const float* mv_dt_grad,
                                                         const float* mv_dt_grad_1, float scale_1,
                                                         const float* dt_image_grad, const float* closest_vertex_id,
                                                         const float* multi_view_crops,
                                                         float* points_image_space_grad) {
    clear_error();
    return sil_backward_run((cudaStream_t)stream, batch, n_cameras, n_points, widths, heights, mv_dt_grad,
                            mv_dt_grad_1, dt_image_grad, closest_vertex_id, multi_view_crops,
                            points_image_space_grad, scale_1);
}

// ---------------------------------------------------------------------------
// No-allocation variant of the silhouette forward.
//
// Some callers cannot call cudaMalloc: a TensorFlow custom op has to take its
// memory from TF's allocator (which already owns most of the device), and
// hosts that pre-allocate everything at start-up forbid allocation on their
// hot path.  This entry point keeps the boundary-vertex grid in a fixed
// file-scope device array instead of the handle's workspace.  The array is
// part of the module image, so every GPU that loads the library holds it
// until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kSilStaticBytes = 8u << 20;  // 8 MiB
static __device__ __align__(256) int g_sil_static[kSilStaticBytes / sizeof(int)];

// The host-side name g_sil_static is not a device address: resolve it once per
// device, with that device current.
hc_status sil_static_base(int** out) {
    static std::mutex mu;
    static std::vector<int*> per_device;
    int dev = 0;
    HC_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if ((int)per_device.size() <= dev) per_device.resize(dev + 1, nullptr);
    if (!per_device[dev]) {
        void* p = nullptr;
        HC_CUDA(cudaGetSymbolAddress(&p, g_sil_static));
        per_device[dev] = static_cast<int*>(p);
    }
    *out = per_device[dev];
    return HC_OK;
}

}  // namespace

extern "C" hc_status hc_silhouette_forward_static(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                                  int32_t resolution_u, int32_t resolution_v,
                                                  const float* points_image_space, const float* normals_image_space,
                                                  const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                                                  const float* multi_view_crops, float* mv_dt_residual,
                                                  float* mv_dt_residual_1, float* dt_image_gradient,
                                                  float* closest_vertex_id) {
    clear_error();
    ImgLayout L;
    size_t need = 0;
    const SameSize sz(n_cameras, resolution_u, resolution_v);
    HC_TRY(sil_forward_plan(batch, n_cameras, n_points, sz.w.data(), sz.h.data(), points_image_space,
                            normals_image_space, is_boundary, distance_transform_image, multi_view_crops,
                            mv_dt_residual, mv_dt_residual_1, dt_image_gradient, closest_vertex_id, L, need));
    HC_REQUIRE(need <= kSilStaticBytes,
               "hc_silhouette_forward_static: %lld views x %d points at %dx%d need %zu bytes of grid scratch; the "
               "static scratch holds %zu bytes (use hc_silhouette_forward)",
               (long long)batch * n_cameras, n_points, resolution_u, resolution_v, need, kSilStaticBytes);
    int* base = nullptr;
    HC_TRY(sil_static_base(&base));
    // the array keeps the previous call's contents: sil_forward_run clears the
    // cell counts before the grid is built
    return sil_forward_run((cudaStream_t)stream, base, L, batch, n_cameras, n_points, points_image_space,
                           normals_image_space, is_boundary, distance_transform_image, multi_view_crops,
                           mv_dt_residual, mv_dt_residual_1, dt_image_gradient, closest_vertex_id);
}
