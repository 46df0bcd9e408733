// Shared state and device helpers of the rasterizer (forward and adjoint).
//
// Layout in HBM (V = B*C views, T = tiles per view):
//   ViewCam   cams[V]             camera set-up, one per view
//   TriFrame  tri_frame[B*F]      per-frame triangle constants (scaled vertices, plane normal)
//   TriView   tri_view[V*F]       per-view triangle constants (ray-plane numerator, pixel bbox)
//   int2      tile_state[V*T]     (binned count, spill slot + 1)
//   int       bins[V*T*CAP]       triangle ids per tile
//   int4      spill[S]            (view, tile, triangle) pairs beyond CAP
//   u64       spill_keys[K*TS*TS] packed (depth_q << 32 | triangle) per spilled tile pixel
#pragma once

#include <vector>

#include "hc_common.cuh"
#include "hc_math.cuh"

namespace hc {

enum AlbedoMode {
    kVertexColor = 0, kTextured, kNormal, kLighting, kForegroundMask, kPosition, kDepth, kUV,
    // bilinear texture sampling (no reference counterpart: the reference's
    // textured mode samples the nearest texel, CUDABasedRasterization.cu:347-373)
    kTexturedBilinear
};
enum ShadingMode { kShaded = 0, kShadeless };
enum NormalMapMode { kNmOriginal = 0, kNmHitPosition, kNmNone, kNmFace };

struct ViewCam {
    float invP[16];  // inverse(K * E), row-major 4x4
    float invE[16];  // inverse(E)
    float ext[12];   // world -> camera, row-major 3x4
    float intr[9];   // row-major 3x3
    float ro[3];     // ray origin (camera centre)
    float ro_s[3];   // ray origin / 1000
    float KE[9];     // K * E[:, :3] (row-major): world -> homogeneous pixel, linear part
    float Kt[3];     // K * E[:, 3]
    // the view's image: resolution, tile grids and where its pixels / tiles
    // start in the call's buffers (cameras of a frame may differ in size)
    int W, H, tiles_x, tiles_x_b;
    long long pix_base, tile_base, tile_base_b;
    FastDiv fd_tiles_x, fd_tiles_x_b;  // division by tiles_x / tiles_x_b
};

constexpr int kAdjointTile = 16;  // tile edge of the renderer adjoint

// One camera's image inside a frame: the frame's cameras are concatenated,
// so views of different resolutions share one launch.
struct CamLayout {
    int W, H;
    int tiles_x, tiles_x_b;        // raster tiles (ws.tile px) / adjoint tiles (16 px) per row
    long long pix, tile, tile_b;   // first pixel / raster tile / adjoint tile in the frame
    FastDiv fd_tiles_x, fd_tiles_x_b;
};

struct TriFrame {    // 48 bytes: s0.xyz n.x | s1.xyz n.y | s2.xyz n.z
    float4 a, b, c;
};

struct TriView {     // 64 bytes per (view, triangle), written by the binning pass
    float num;       // dot(s0, n) - dot(ro_s, n)
    int x01;         // bbox x0 | x1 << 16
    int y01;         // bbox y0 | y1 << 16
    int dqmin;       // lower bound of the quantised depth; bit 31 set = back-facing
    float4 e01;      // 2-D footprint edges 0 and 1: (a0, b0, a1, b1)
    float4 e2c;      // edge 2 and two offsets: (a2, b2, c0, c1)
    float4 e2o;      // (c2, 0, 0, 0)
};

struct TriS;


struct RasterStats {
    unsigned long long binned;
    unsigned long long spilled;
    int spill_tiles;
    int overflow;      // bit 0: spill list full, bit 1: spill tile slots exhausted,
                       // bit 2: an adjoint target copy (TMA) did not complete
};

// Pixel-centre camera ray (reference getRayCuda2 / backprojectPixelCuda,
// CudaRenderer/cpp/src/Utils/CameraUtil.h:223-258): the pixel centre is lifted
// to depth 1000 through inv(K*E) and the direction from the camera centre is
// normalised with rsqrtf.
__device__ __forceinline__ float3 pixel_ray(const ViewCam& c, int px, int py) {
    const float u = px + 0.5f;
    const float v = py + 0.5f;
    const float4 tp = make_float4(u * 1000.f, v * 1000.f, 1000.f, 1.f);
    const float4 r0 = make_float4(c.invP[0], c.invP[1], c.invP[2], c.invP[3]);
    const float4 r1 = make_float4(c.invP[4], c.invP[5], c.invP[6], c.invP[7]);
    const float4 r2 = make_float4(c.invP[8], c.invP[9], c.invP[10], c.invP[11]);
    const float3 q = make_float3(dot(r0, tp), dot(r1, tp), dot(r2, tp));
    return normalize3(q - make_float3(c.ro[0], c.ro[1], c.ro[2]));
}

struct TriS {
    float3 s0, s1, s2, n;
};

__device__ __forceinline__ TriS tri_from(const TriFrame& f) {
    TriS t;
    t.s0 = make_float3(f.a.x, f.a.y, f.a.z);
    t.s1 = make_float3(f.b.x, f.b.y, f.b.z);
    t.s2 = make_float3(f.c.x, f.c.y, f.c.z);
    t.n = make_float3(f.a.w, f.b.w, f.c.w);
    return t;
}

// Conservative lower bound of int(t * 1e4) over the triangle.  For a unit
// ray direction t is the distance from the camera centre to the hit point,
// which is at least (a) the distance to the triangle's plane, |num| / |n|,
// and (b) the distance to the nearest vertex minus the longest edge (every
// point of a triangle lies within its longest edge of some vertex).  The
// larger of the two is lowered by 1e-4 relative and 2 quanta so float
// rounding of either side cannot break it.
__device__ __forceinline__ int depth_lower_bound(float num, float3 n, const TriS& T, float3 o) {
    const float pd = fabsf(num) / sqrtf(dot(n, n));
    // the minimum / maximum taken on the squared lengths and rooted once: the
    // correctly rounded square root is monotone, so the values are those of
    // the per-vertex and per-edge lengths
    const float3 a0 = T.s0 - o, a1 = T.s1 - o, a2 = T.s2 - o;
    const float dmin = sqrtf(fminf(dot(a0, a0), fminf(dot(a1, a1), dot(a2, a2))));
    const float3 e0 = T.s1 - T.s0, e1 = T.s2 - T.s1, e2 = T.s0 - T.s2;
    const float e = sqrtf(fmaxf(dot(e0, e0), fmaxf(dot(e1, e1), dot(e2, e2))));
    const float vd = dmin - e;
    const float z = fmaxf(pd, vd) * 10000.f * (1.f - 1e-4f);
    if (!(z < 2.0e9f)) return 0x7fffffff;
    return max((int)z - 2, 0);
}

// Ray / triangle test of the reference (rayTriangleIntersect,
// CudaRenderer/cpp/src/Utils/RendererUtil.h:26-101) with the per-triangle and
// per-view terms hoisted: s* = vertices / 1000, n = cross(s1 - s0, s2 - s0),
// num = dot(s0, n) - dot(origin / 1000, n).  Same operations in the same order
// per pixel, so hit decisions, t and the barycentrics (a weights s0, b weights
// s1) match the reference bit for bit.
__device__ __forceinline__ bool ray_tri(float3 ro_s, float3 dir, const TriS& T, float num,
                                        float& t, float& a, float& b) {
    const float ndr = dot(dir, T.n);
    if (fabsf(ndr) < 0.0000001f) return false;
    t = num / ndr;
    if (t < 0.f) return false;
    const float3 P = ro_s + t * dir;
    float3 C = cross(T.s1 - T.s0, P - T.s0);
    if (dot(T.n, C) < 0.f) return false;
    C = cross(T.s2 - T.s1, P - T.s1);
    if ((a = dot(T.n, C)) < 0.f) return false;
    C = cross(T.s0 - T.s2, P - T.s2);
    if ((b = dot(T.n, C)) < 0.f) return false;
    const float denom = dot(T.n, T.n);
    a /= denom;
    b /= denom;
    return true;
}

// Barycentrics of a pixel's known winner: the operations of ray_tri that
// form a and b, without the sign and window checks that the winner has
// passed (so the values are ray_tri's).
__device__ __forceinline__ void winner_bary(float3 ro_s, float3 dir, const TriS& T, float num, float& a, float& b) {
    const float ndr = dot(dir, T.n);
    const float t = num / ndr;
    const float3 P = ro_s + t * dir;
    float3 C = cross(T.s2 - T.s1, P - T.s1);
    a = dot(T.n, C);
    C = cross(T.s0 - T.s2, P - T.s2);
    b = dot(T.n, C);
    const float denom = dot(T.n, T.n);
    a /= denom;
    b /= denom;
}

// Hit accepted by the depth pass: barycentric window of
// CUDABasedRasterization.cu:243 and the quantised depth int(t * 1e4) of :247-250.
__device__ __forceinline__ bool raster_hit(float3 ro_s, float3 dir, const TriS& T, float num,
                                           int& depth_q, float& a, float& b) {
    float t;
    if (!ray_tri(ro_s, dir, T, num, t, a, b)) return false;
    if (!((a >= -0.001f) && (b >= -0.001f) && (a <= 1.001f) && (b <= 1.001f))) return false;
    depth_q = (int)(t * 10000.f);
    return true;
}

// World -> camera -> pixel projection (reference getCamSpacePoint and
// projectPointFloat3, CudaRenderer/cpp/src/Utils/CameraUtil.h:141-186).
__device__ __forceinline__ float3 project_point(const float* ext, const float* intr, float3 p) {
    const float4 h = make_float4(p.x, p.y, p.z, 1.f);
    const float3 cs = make_float3(dot(make_float4(ext[0], ext[1], ext[2], ext[3]), h),
                                  dot(make_float4(ext[4], ext[5], ext[6], ext[7]), h),
                                  dot(make_float4(ext[8], ext[9], ext[10], ext[11]), h));
    const float3 d1 = cs * make_float3(intr[0], intr[1], intr[2]);
    const float3 d2 = cs * make_float3(intr[3], intr[4], intr[5]);
    const float3 d3 = cs * make_float3(intr[6], intr[7], intr[8]);
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
    return make_float3(x, y, z);
}

// Conservative 2-D footprint of a triangle in a view: the three edge lines of
// its projection, each widened by a margin, as signed pixel distances that
// are non-negative inside.  A pixel centre outside the widened triangle
// cannot pass the exact test that follows:
//  * the ray test: for vertices in front of the camera the projected
//    triangle is the exact image of the 3-D one, and the float error of
//    either computation is below 1e-3 px for the coordinate ranges admitted
//    here (|u|, |v| < 1e5 px, z > 1), against a margin of kEdgeMargin px;
//  * the image-space barycentric test with its -0.001 tolerance: edge k is
//    additionally widened by 0.0011 x the triangle's height over that edge,
//    and by num_err / |edge k| px, num_err bounding the rounding error of
//    that test's edge-function numerator (2e-6 M^2 for coordinates up to M).
// Outside that coordinate range, or for a projected area under 1e-2 px^2, the
// footprint is disabled (every pixel passes).  It only skips work; it never
// decides a hit.
constexpr float kEdgeMargin = 0.125f;

struct Footprint {
    float a[3], b[3], c[3];  // edge k: a*x + b*y + c >= 0 inside (margin included)
    float m[3];              // the margin folded into c[k] (0 when disabled)
};
// A pixel centre whose three footprint values are all >= kEdgeInterior lies
// inside the (unwidened) projected triangle by more than kEdgeMargin px: the
// exact ray test's edge and barycentric-window checks certainly pass there.
// (A disabled footprint has values 0 and never qualifies.)
constexpr float kEdgeInterior = 2.f * kEdgeMargin;

__device__ __forceinline__ Footprint footprint(float3 p0, float3 p1, float3 p2, float rel_margin = 0.f,
                                               float num_err = 0.f) {
    Footprint fp;
    const float3 q[3] = {p0, p1, p2};
    bool ok = p0.z > 1.f && p1.z > 1.f && p2.z > 1.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) ok = ok && fabsf(q[k].x) < 1e5f && fabsf(q[k].y) < 1e5f;
    const float area = (p1.x - p0.x) * (p2.y - p0.y) - (p1.y - p0.y) * (p2.x - p0.x);
    ok = ok && fabsf(area) >= 1e-2f;
    const float sg = area > 0.f ? 1.f : -1.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float3 u = q[k], w = q[(k + 1) % 3];
        const float ex = w.x - u.x, ey = w.y - u.y;
        const float len = sqrtf(ex * ex + ey * ey);
        if (!(len > 1e-6f)) ok = false;
        const float inv = ok ? sg / len : 0.f;
        // (the widenings are skipped when both are zero: 0 / len is not
        // folded away by the compiler, and adds nothing)
        const bool widen = ok && (rel_margin != 0.f || num_err != 0.f);
        const float margin = kEdgeMargin + (widen ? rel_margin * fabsf(area) / len + num_err / len : 0.f);
        // signed distance of (x, y) from the edge u -> w, positive on the inside
        fp.a[k] = -ey * inv;
        fp.b[k] = ex * inv;
        fp.c[k] = (ey * u.x - ex * u.y) * inv + margin;
        fp.m[k] = ok ? margin : 0.f;
    }
    if (!ok) {  // disabled: every pixel is on the boundary band (passes, never "inside")
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            fp.a[k] = 0.f;
            fp.b[k] = 0.f;
            fp.c[k] = 0.f;
            fp.m[k] = 0.f;
        }
    }
    return fp;
}

// false when no pixel centre of [x0, x1] x [y0, y1] can be inside the footprint
__device__ __forceinline__ bool footprint_overlaps(const Footprint& fp, int x0, int x1, int y0, int y1) {
    const float xa = x0 + 0.5f, xb = x1 + 0.5f, ya = y0 + 0.5f, yb = y1 + 0.5f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float m = fp.a[k] * (fp.a[k] > 0.f ? xb : xa) + fp.b[k] * (fp.b[k] > 0.f ? yb : ya) + fp.c[k];
        if (m < 0.f) return false;
    }
    return true;
}

// Bilinear texture lookup at texel coordinates (x, y), texel centres at
// integer + 0.5, clamp-to-edge addressing: the four texel offsets (floats,
// x3 channels) and weights.
struct BilinearTaps {
    long long o00, o10, o01, o11;
    float fx, fy;
};

__device__ __forceinline__ BilinearTaps bilinear_taps(float x, float y, int tw, int th) {
    const float sx = x - 0.5f, sy = y - 0.5f;
    const float x0f = floorf(sx), y0f = floorf(sy);
    BilinearTaps t;
    t.fx = sx - x0f;
    t.fy = sy - y0f;
    const int x0 = (int)x0f, y0 = (int)y0f;
    const int xa = min(max(x0, 0), tw - 1), xb = min(max(x0 + 1, 0), tw - 1);
    const int ya = min(max(y0, 0), th - 1), yb = min(max(y0 + 1, 0), th - 1);
    t.o00 = 3LL * ((long long)ya * tw + xa);
    t.o10 = 3LL * ((long long)ya * tw + xb);
    t.o01 = 3LL * ((long long)yb * tw + xa);
    t.o11 = 3LL * ((long long)yb * tw + xb);
    return t;
}

__device__ __forceinline__ float3 bilinear_sample(const float* T, const BilinearTaps& t) {
    const float3 c00 = ld3(T + t.o00), c10 = ld3(T + t.o10), c01 = ld3(T + t.o01), c11 = ld3(T + t.o11);
    const float w00 = (1.f - t.fx) * (1.f - t.fy), w10 = t.fx * (1.f - t.fy), w01 = (1.f - t.fx) * t.fy,
                w11 = t.fx * t.fy;
    return c00 * w00 + c10 * w10 + c01 * w01 + c11 * w11;
}

// Second-order SH shading of an albedo (reference getShading,
// CudaRenderer/cpp/src/Utils/RendererUtil.h:135-173), one band set per channel.
__device__ __forceinline__ float sh_channel(const float* s, float3 d, float3 d2) {
    float r = s[0];
    r += s[1] * d.y;
    r += s[2] * d.z;
    r += s[3] * d.x;
    r += s[4] * (d.x * d.y);
    r += s[5] * (d.z * d.y);
    r += s[6] * (3.f * d2.z - 1.f);
    r += s[7] * (d.x * d.z);
    r += s[8] * (d2.x - d2.y);
    return r;
}

__device__ __forceinline__ float3 sh_illum(const float* sh, float3 n) {
    const float3 n2 = n * n;
    return make_float3(sh_channel(sh, n, n2), sh_channel(sh + 9, n, n2), sh_channel(sh + 18, n, n2));
}

struct Topology {
    int N = 0, F = 0;
    DevBuf faces;        // int3[F]
    DevBuf vf;           // int[3F]  vertex -> faces, increasing face id
    DevBuf vf_id;        // int2[N]  (start, count)
    DevBuf texcoords;    // float[6F]
    bool has_texcoords = false;
};

// texel -> (face, barycentrics) table of the UV-space maps, per texture size
struct UvTable {
    int th = 0, tw = 0;
    DevBuf faces, table;
};

// Optional per-kernel timing of the renderer (CUDA events around each
// launch on the launching stream), for benchmarks; off by default.
enum RendererKernel {
    kKViewSetup = 0, kKVertexNormals, kKTriFrame, kKBin, kKSpill, kKResolve, kKRenderGrad, kKNormalChain,
    kKCount
};

struct KernelClock {
    bool on = false, made = false;
    cudaEvent_t ev[2 * kKCount];
    unsigned recorded = 0;  // kernels with both events recorded since the last read
    void begin(int k, cudaStream_t s) {
        if (on) cudaEventRecord(ev[2 * k], s);
    }
    void end(int k, cudaStream_t s) {
        if (!on) return;
        cudaEventRecord(ev[2 * k + 1], s);
        recorded |= 1u << k;
    }
};

// The masked image L1 fused into the raster (hc_renderer_forward_l1 /
// hc_renderer_backward_l1): the forward's tile pass accumulates the loss of
// the pixels it shades, the adjoint forms the image gradient inline instead
// of reading it.
struct L1Fuse {
    const float* target = nullptr;        // [B, P_frame, 3]
    const unsigned char* mask = nullptr;  // [B, P_frame] foreground mask, or NULL
    L1State* state = nullptr;             // written by the forward, read by the adjoint
    float* loss = nullptr;                // forward: sum / count, or NULL
    const float* render = nullptr;        // adjoint: the forward's render buffer
};

struct RasterWorkspace {
    int cap_views = 0;   // views the buffers are sized for
    int tile = 16;
    int bin_cap = 512;
    // per-camera resolution and the device layout derived from it
    std::vector<int> cam_w, cam_h;
    int layout_tile = 0;                              // tile size the layout was built for
    long long P_frame = 0, T_frame = 0, Tb_frame = 0; // pixels / raster tiles / adjoint tiles per frame
    DevBuf layout, tile_cam, tile_cam_b;              // CamLayout[C]; camera of each tile of a frame
    long long spill_cap = 0;
    int spill_tile_cap = 0;
    DevBuf cams, tri_frame, tri_view, tile_state, bins, spill, spill_keys, stats;
    DevBuf proj;  // float4 [V,N]: projected vertices of the current call
    DevBuf l1_part;  // per raster tile: float L1 sum, unsigned count (fused L1 only)
    DevBuf claim;    // the tile resolve's tile counter
    DevBuf claim_b;  // the adjoint's tile counter
    int adjoint_dynamic = 1;  // the adjoint's tile schedule (hc_renderer_set_adjoint_schedule)
    KernelClock clock;
};

}  // namespace hc
