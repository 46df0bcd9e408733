// Renderer adjoint (the CudaRendererGradGpu op).
//
// Reference: CudaRenderer/cpp/src/Renderer/CUDABasedRasterizationGrad.cu:114-496
// with the Jacobians of CudaRenderer/cpp/src/Utils/RendererUtil.h:241-914.
// There, one thread per pixel scatters 9 position + 9 colour + 27 SH float
// atomics to global memory, and in shaded mode loops over every face around
// each of its three vertices (another ~160 atomics per pixel).  Here:
//  * one CTA per 16x16 pixel tile, the target image tile (+ filter halo)
//    staged in shared memory for the image-gradient taps;
//  * the barycentric Jacobian is the exact rank-1 form (below) instead of the
//    reference's 3x9 product (which is kept as the parity mode);
//  * per-vertex contributions (position, colour, pixel-normal gradients) are
//    merged inside each warp (lanes matched by face id, a leader sums up to
//    8 members) before one global reduction per vertex and leader;
//  * SH gradients are reduced over the CTA (warp shuffles) before one atomic
//    per coefficient;
//  * the shaded-mode normal chain is split in two: pixels accumulate the
//    gradient w.r.t. each vertex's unnormalised normal, then a per-vertex
//    gather over incident faces applies d(face normal)/d(vertex) once per
//    frame (same sum as the reference's per-pixel loops, reassociated).
#include <algorithm>

#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched through the runtime)

#include "renderer.cuh"

namespace hc {

__global__ void k_view_setup(int V, int C, const float* __restrict__ extr, const float* __restrict__ intr,
                             const CamLayout* __restrict__ layout, long long P_frame, long long T_frame,
                             long long Tb_frame, ViewCam* __restrict__ cams);

namespace {

constexpr int BT = 16;           // backward tile edge
constexpr int BNT = BT * BT;     // threads per CTA
static_assert(BT == kAdjointTile, "the adjoint tile grid of the layout");

struct BwdArgs {
    int B, C, N, F;
    long long Tb_frame;      // adjoint tiles per frame (all cameras)
    FastDiv fd_frame;        // division by Tb_frame (the call has < 2^31 adjoint tiles)
    FastDiv fd_est;          // division by the staged tile edge BT + 2 ifs
    const int* tile_cam_b;   // camera of each adjoint tile of a frame
    int albedo, shading;
    int ifs, tfs;
    int tex_w, tex_h;
    const int3* faces;
    const float* texcoords;
    const float* grad;      // [V,H,W,3]
    const float* verts;     // [B,N,3]
    const float* colors;    // [B,N,3]
    const float* texture;   // [B,TH,TW,3]
    const float* sh;        // [V,27]
    const float* target;    // [V,H,W,3]
    const float* vnormal;   // [V,N,3]
    const float* bary;      // [V,H,W,2]
    const int* face;        // [V,H,W]
    float* vpos_grad;       // [B,N,3]
    float* vcol_grad;       // [B,N,3]
    float* tex_grad;        // [B,TH,TW,3]
    float* sh_grad;         // [V,27]
    float* nrm_grad;        // [B,N,3] workspace: d loss / d (unnormalised vertex normal)
    // fused image L1: the image gradient is formed from the render and the
    // target instead of read from grad (NULL state: not fused)
    const L1State* l1_state;
    const float* l1_render;          // [V,H,W,3]
    int* err;                        // bit 2: a target copy did not complete (RasterStats::overflow)
    unsigned* claim;                 // tile counter of the persistent CTAs (cleared before the launch)
    const unsigned char* l1_mask;    // [V,H,W] or NULL
};

__device__ __forceinline__ float3 unit3(int k) {
    return make_float3(k == 0 ? 1.f : 0.f, k == 1 ? 1.f : 0.f, k == 2 ? 1.f : 0.f);
}

// d(a, b)/d(v0, v1, v2): the barycentric Jacobian of the reference's
// dJBCDVerpos (RendererUtil.h:670-861) for a = dot(N, C1)/|N|^2 (weight of
// v0) and b = dot(N, C2)/|N|^2 (weight of v1), in unscaled (mm) coordinates,
// contracted with the gradient w.r.t. the three barycentrics as it is formed:
// gp[var] = g.x * ja[var] + g.y * jb[var] + g.z * (-ja[var] - jb[var]), the
// reference's 3x9 product, one column at a time (no 2 x 9 row arrays live).
// Leaves gp at zero for grazing rays or degenerate triangles.
__device__ __forceinline__ void bary_jacobian_apply(float3 o, float3 d, float3 v0, float3 v1, float3 v2, float3 g,
                                                    float gp[9]) {
    const float3 e01 = v1 - v0, e02 = v2 - v0;
    const float3 N = cross(e01, e02);
    const float denom = dot(N, N);
    const float ndr = dot(d, N);
#pragma unroll
    for (int i = 0; i < 9; ++i) gp[i] = 0.f;
    if (fabsf(dot(normalize3(d), normalize3(N))) < 0.001f || fabsf(denom * denom) < 0.001f) return;
    const float t = (dot(v0, N) - dot(o, N)) / ndr;
    const float3 P = o + t * d;
    const float3 E0 = v2 - v1, E1 = v0 - v2;
    const float3 vp0 = P - v1, vp1 = P - v2;
    const float3 C0 = cross(E0, vp0), C1 = cross(E1, vp1);
    const float tmp0 = dot(N, C0), tmp1 = dot(N, C1);
    const float3 v0mo = v0 - o;
    const float v0moN = dot(v0mo, N);
    const float inv_ndr = 1.f / ndr;
    const float inv_ndr2 = -1.f / (ndr * ndr);
    const float inv_den = 1.f / denom;
    const float inv_den2 = -1.f / (denom * denom);
#pragma unroll
    for (int var = 0; var < 9; ++var) {
        const int vert = var / 3;
        const float3 ek = unit3(var % 3);
        const float3 z = make_float3(0.f, 0.f, 0.f);
        float3 dN;
        if (vert == 0) dN = cross(-ek, e02) + cross(e01, -ek);
        else if (vert == 1) dN = cross(ek, e02);
        else dN = cross(e01, ek);
        const float3 dv0 = vert == 0 ? ek : z;
        const float3 dv1 = vert == 1 ? ek : z;
        const float3 dv2 = vert == 2 ? ek : z;
        const float dt = inv_ndr2 * dot(dN, d) * v0moN + inv_ndr * (dot(dv0, N) + dot(v0mo, dN));
        const float3 dE0 = dv2 - dv1, dE1 = dv0 - dv2;
        const float nd = 2.f * dot(N, dN);
        const float dtmp0 = dot(dN, C0) + dot(N, cross(dE0, vp0) + cross(E0, dt * d - dv1));
        const float dtmp1 = dot(dN, C1) + dot(N, cross(dE1, vp1) + cross(E1, dt * d - dv2));
        const float ja = dtmp0 * inv_den + tmp0 * inv_den2 * nd;
        const float jb = dtmp1 * inv_den + tmp1 * inv_den2 * nd;
        gp[var] = g.x * ja + g.y * jb + g.z * (-ja - jb);
    }
}

// Sobel-like image gradient of the reference (imageGradient, RendererUtil.h:566-620):
// weights (x, y)/(x^2+y^2) over a (2k+1)^2 window, normalised by sum |x|/(x^2+y^2);
// zero near the border.  `x`, `y` are the (possibly fractional) sample position.
__device__ void image_gradient(const float* img, float x, float y, int w, int h, int fs, float3& du, float3& dv) {
    du = dv = make_float3(0.f, 0.f, 0.f);
    if (!(x >= (float)(fs + 1) && y >= (float)(fs + 1) && x < (float)(w - (fs + 1)) && y < (float)(h - (fs + 1))))
        return;
    float norm = 0.f;
    for (int j = -fs; j <= fs; ++j)
        for (int i = -fs; i <= fs; ++i) {
            const int idx = (int)((y + j) * w + (x + i));
            const float3 I = ld3(img + 3LL * idx);
            const float den = (float)(i * i + j * j);
            float gu = 0.f, gv = 0.f;
            if (den != 0.f) {
                gu = (float)i / den;
                gv = (float)j / den;
            }
            du += I * gu;
            dv += I * gv;
            norm += fabsf(gu);
        }
    du = du / norm;
    dv = dv / norm;
}

// Exact barycentric Jacobian of a ray hit.  With P = o + t d = l0 v0 + l1 v1 +
// l2 v2 (l2 = 1 - l0 - l1), perturbing vertex i moves (t, l0, l1) by
// l_i M^-1 dv_i with M = [d, -(v0 - v2), -(v1 - v2)], so
//   d l0 / d v_i = l_i (d x (v1 - v2)) / (d . N),
//   d l1 / d v_i = l_i ((v0 - v2) x d) / (d . N),   N = (v1 - v0) x (v2 - v0).
// Same function as the reference's dJBCDVerpos (RendererUtil.h:670-861) in
// exact arithmetic, without the intersection point (better conditioned).
// Returns false for the reference's grazing / degenerate cut-off.
__device__ __forceinline__ bool bary_rows(float3 d, float3 v0, float3 v1, float3 v2, float3& r0, float3& r1) {
    const float3 N = cross(v1 - v0, v2 - v0);
    const float denom = dot(N, N);
    if (fabsf(dot(normalize3(d), normalize3(N))) < 0.001f || fabsf(denom * denom) < 0.001f) return false;
    const float inv = 1.f / dot(d, N);
    r0 = cross(d, v1 - v2) * inv;
    r1 = cross(v0 - v2, d) * inv;
    return true;
}

constexpr int MAXFS = 4;                 // image filter sizes staged in shared memory
constexpr int TILE_S = BT + 2 * MAXFS;   // staged target tile edge

constexpr int MAXTAPS = (2 * MAXFS + 1) * (2 * MAXFS + 1);
// TMA staging: one box of rows x kRawX floats of the target viewed as
// [views][H][3W], its x start rounded down to 16 bytes
constexpr int kRawX = (3 * TILE_S + 3 + 3) / 4 * 4;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_try_wait(unsigned mbar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(mbar), "r"(parity)
                 : "memory");
    return ok != 0;
}

// a bounded wait: false when the phase did not complete within the limit
__device__ __forceinline__ bool mbar_wait(unsigned mbar, unsigned parity) {
    for (int k = 0; k < (1 << 20); ++k)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

// one thread: expect the box's bytes on the barrier and start the tensor copy
__device__ __forceinline__ void tma_box(const CUtensorMap* map, unsigned dst, unsigned mbar, int x, int y, int z,
                                        unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}

// G . dTarget/d(u, v) over the staged (2 FS + 1)^2 window for a compile-time
// filter size: the weights (i, j) / (i^2 + j^2) fold to the same correctly
// rounded constants the per-CTA table holds, and the taps are summed in the
// same (row, column) order, leaving out only terms that are exact zeros, so
// both paths give identical results for finite targets.
template <int FS>
__device__ __forceinline__ void taps_fs(const float4* s_tgt, int s0, float3 G, float& gu, float& gv) {
    constexpr int e = BT + 2 * FS;
#pragma unroll
    for (int j = -FS; j <= FS; ++j)
#pragma unroll
        for (int i = -FS; i <= FS; ++i) {
            // the centre has no weight and the zero weights add exact zeros
            // (the sums start at +0 and stay finite), so they are skipped
            if (i == 0 && j == 0) continue;
            const float den = (float)(i * i + j * j);
            const float wi = (float)i / den, wj = (float)j / den;
            const float4 I = s_tgt[s0 + (j + FS) * e + (i + FS)];
            const float gi = G.x * I.x + G.y * I.y + G.z * I.z;
            if (i != 0) gu += gi * wi;
            if (j != 0) gv += gi * wj;
        }
}

// Albedo classes of the adjoint: vertex colours, texture, and the modes
// whose albedo has no parameters (normal, lighting, mask, position, depth, uv).
enum { kAlbVcol = 0, kAlbTex = 1, kAlbNone = 2, kAlbTexBilinear = 3 };

template <bool SHADED, int ALB, bool PARITY, bool DYN>
__global__ void __launch_bounds__(BNT, SHADED ? 2 : 4) k_render_grad(BwdArgs A, const ViewCam* __restrict__ cams, long long n_tiles,
                                                                     const __grid_constant__ CUtensorMap tmap,
                                                                     int use_tma) {
    constexpr int NVV = SHADED ? 9 : 6;               // values per vertex
    constexpr int NROW = (3 * NVV + 3) / 4 * 4;       // per-lane row, padded for float4 loads
    __shared__ __align__(16) float s_red[BNT / 32][32][NROW];
    __shared__ float s_sh[SHADED ? BNT / 32 : 1][27];
    __shared__ __align__(128) float4 s_tgt2[2][TILE_S * TILE_S];  // target tile + halo, double-buffered
    __shared__ float2 s_tap[MAXTAPS];  // image-gradient tap weights (i, j) / (i^2 + j^2)
    __shared__ float s_norm;
    __shared__ __align__(8) unsigned long long s_mbar;
    constexpr bool shaded = SHADED;
    constexpr bool vcol = ALB == kAlbVcol;
    constexpr bool textured = ALB == kAlbTex;
    constexpr bool bilinear = ALB == kAlbTexBilinear;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool staged = A.ifs <= MAXFS;
    float l1_scale = 0.f;  // 255 / count of the fused L1
    if (A.l1_state) {
        const unsigned long long cnt = A.l1_state->count;
        l1_scale = cnt ? 255.f / (float)cnt : 0.f;
    }
    if (staged) {
        // tap weights and their normaliser, once per CTA: the same divisions
        // and the same summation order as evaluating them per pixel
        const int fs = A.ifs, ew = 2 * fs + 1;
        if (threadIdx.x < ew * ew) {
            const int i = (int)threadIdx.x % ew - fs, j = (int)threadIdx.x / ew - fs;
            const float den = (float)(i * i + j * j);
            s_tap[threadIdx.x] = den == 0.f ? make_float2(0.f, 0.f) : make_float2((float)i / den, (float)j / den);
        }
        if (threadIdx.x == 0) {
            float norm = 0.f;
            for (int j = -fs; j <= fs; ++j)
                for (int i = -fs; i <= fs; ++i) {
                    const float den = (float)(i * i + j * j);
                    if (den != 0.f) norm += fabsf((float)i / den);
                }
            s_norm = norm;
        }
    }
    // Persistent CTAs walk the 16x16 tiles of the call (the frame's cameras
    // concatenated).  The target tile + filter halo of the next tile is
    // copied into the other shared buffer with cp.async while this tile's
    // pixels are processed, so the copy latency is hidden.
    auto stage = [&](long long gt, int buf) {
        const unsigned sb = A.fd_frame.div((unsigned)gt);
        const ViewCam& sc = cams[(int)sb * A.C + A.tile_cam_b[A.fd_frame.mod((unsigned)gt, sb)]];
        const int st = (int)(gt - sc.tile_base_b);
        const int sty = (int)sc.fd_tiles_x_b.div((unsigned)st);
        const int sx0 = (int)sc.fd_tiles_x_b.mod((unsigned)st, sty) * BT, sy0 = sty * BT;
        const float* stg = A.target + sc.pix_base * 3;
        const int e = BT + 2 * A.ifs;
        for (int i = threadIdx.x; i < e * e; i += BNT) {
            const int yy = sy0 - A.ifs + i / e, xx = sx0 - A.ifs + i % e;
            if (xx >= 0 && yy >= 0 && xx < sc.W && yy < sc.H) {
                const float* src = stg + 3 * ((long long)yy * sc.W + xx);
                const unsigned dst = (unsigned)__cvta_generic_to_shared(&s_tgt2[buf][i]);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src));
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + 4), "l"(src + 1));
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst + 8), "l"(src + 2));
            } else {
                s_tgt2[buf][i] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    };
    // TMA mode (all cameras of one size, rows of 16-byte multiples): one
    // tensor copy per tile of the target box [rows][kRawX] into s_raw,
    // completing on s_mbar, issued while the previous tile is processed and
    // spread into the tap layout when its tile starts.
    const bool tma = use_tma && staged;
    // TMA mode: the tap layout lives in s_tgt2[0] and the box of the next
    // tile in s_tgt2[1] (TILE_S x kRawX floats fit in TILE_S^2 float4)
    static_assert(TILE_S * kRawX <= 4 * TILE_S * TILE_S, "the TMA box fits the second buffer");
    float* const s_raw = reinterpret_cast<float*>(s_tgt2[1]);
    const int e_st = BT + 2 * A.ifs;
    const unsigned raw_bytes = (unsigned)(e_st * kRawX * sizeof(float));
    auto tma_issue = [&](long long gt) {  // thread 0
        const unsigned sb = A.fd_frame.div((unsigned)gt);
        const int sv = (int)sb * A.C + A.tile_cam_b[A.fd_frame.mod((unsigned)gt, sb)];
        const ViewCam& sc = cams[sv];
        const int st = (int)(gt - sc.tile_base_b);
        const int sty = (int)sc.fd_tiles_x_b.div((unsigned)st);
        const int x = (3 * ((int)sc.fd_tiles_x_b.mod((unsigned)st, sty) * BT - A.ifs)) & ~3;  // floats, rounded down to 16 bytes
        const int y = sty * BT - A.ifs;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tma_box(&tmap, smem_u32(s_raw), smem_u32(&s_mbar), x, y, sv, raw_bytes);
    };
    // Tiles are taken one ahead (the next tile's target copy is issued while
    // this one is processed).  DYN: the CTAs claim tiles from a counter, so
    // tiles of uneven cost balance and a CTA that starts late takes fewer
    // (thread 0 writes the ring slot of the next iteration; a barrier
    // separates every write of a slot from its reads).  Static: CTA i takes
    // tiles i, i + grid, ..., and CTAs that run out early free their SM for
    // concurrent work.
    __shared__ int s_claimed[2];
    if (threadIdx.x == 0) {
        if constexpr (DYN) s_claimed[0] = (int)atomicAdd(A.claim, 1u);
        if (tma) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    if (DYN || tma) __syncthreads();
    long long g;
    if constexpr (DYN) g = s_claimed[0];
    else g = blockIdx.x;
    if (tma) {
        if (threadIdx.x == 0 && g < n_tiles) tma_issue(g);
    } else if (staged && g < n_tiles) {
        stage(g, 0);
    }
    asm volatile("cp.async.commit_group;\n" ::);
    for (int it = 0; g < n_tiles; ++it) {  // CTA-uniform
    const int buf = tma ? 0 : it & 1;
    const float4* s_tgt = s_tgt2[buf];
    if (tma) {
        // this tile's box: wait (bounded), spread it into the tap layout, then
        // start the next tile's copy into the freed box
        const bool ok = __syncthreads_and(mbar_wait(smem_u32(&s_mbar), (unsigned)(it & 1)));
        if (!ok) {  // the copy did not land: flag it, give it one more bounded wait, stop
            if (threadIdx.x == 0) atomicOr(A.err, 4);
            mbar_wait(smem_u32(&s_mbar), (unsigned)(it & 1));
            return;
        }
        const unsigned gb = A.fd_frame.div((unsigned)g);
        const ViewCam& gc = cams[(int)gb * A.C + A.tile_cam_b[A.fd_frame.mod((unsigned)g, gb)]];
        const unsigned gtile = (unsigned)(g - gc.tile_base_b);
        const int cx0 = (int)gc.fd_tiles_x_b.mod(gtile, gc.fd_tiles_x_b.div(gtile)) * BT - A.ifs;
        const int off = 3 * cx0 - ((3 * cx0) & ~3);  // floats before the first halo column in a box row
        for (int i = threadIdx.x; i < e_st * e_st; i += BNT) {
            const int r = (int)A.fd_est.div((unsigned)i), c = i - r * e_st;
            const float* q = s_raw + r * kRawX + off + 3 * c;
            s_tgt2[buf][i] = make_float4(q[0], q[1], q[2], 0.f);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long nx;
            if constexpr (DYN) {
                nx = atomicAdd(A.claim, 1u);
                s_claimed[(it + 1) & 1] = (int)nx;
            } else {
                nx = g + gridDim.x;
            }
            if (nx < n_tiles) tma_issue(nx);
        }
    } else {
        long long nx;
        if constexpr (DYN) {
            if (threadIdx.x == 0) s_claimed[(it + 1) & 1] = (int)atomicAdd(A.claim, 1u);
            __syncthreads();  // every thread stages the next tile
            nx = s_claimed[(it + 1) & 1];
        } else {
            nx = g + gridDim.x;
        }
        if (staged && nx < n_tiles) stage(nx, buf ^ 1);
    }
    asm volatile("cp.async.commit_group;\n" ::);
    const unsigned fb = A.fd_frame.div((unsigned)g);
    const int b = (int)fb;
    const int view = b * A.C + A.tile_cam_b[A.fd_frame.mod((unsigned)g, fb)];
    const ViewCam& cam = cams[view];
    const int tile = (int)(g - cam.tile_base_b);
    const int W = cam.W, H = cam.H;
    const int tyi = (int)cam.fd_tiles_x_b.div((unsigned)tile);
    const int tx0 = (int)cam.fd_tiles_x_b.mod((unsigned)tile, tyi) * BT, ty0 = tyi * BT;
    const int px = tx0 + threadIdx.x % BT;
    const int py = ty0 + threadIdx.x / BT;
    const float* tgt = A.target + cam.pix_base * 3;
    float shg[SHADED ? 27 : 1];
#pragma unroll
    for (int k = 0; k < (SHADED ? 27 : 1); ++k) shg[k] = 0.f;
    const long long pix = cam.pix_base + (long long)py * W + px;
    const int f = (px < W && py < H) ? A.face[pix] : -1;
    int vid[3] = {-1, -1, -1};
    float bw[3] = {0.f, 0.f, 0.f};
    float gp[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) gp[k] = 0.f;
    float3 gA = make_float3(0.f, 0.f, 0.f), gnu = make_float3(0.f, 0.f, 0.f);
    // carried from the first half of the pixel work to the second (with cp.async
    // staging the first half reads no staged target: its copies are in flight)
    float3 d = make_float3(0.f, 0.f, 1.f), v0 = d, v1 = d, v2 = d, G = d, frag = d;
    float3 gbc = make_float3(0.f, 0.f, 0.f);  // d loss / d (a, b, c)
    if (f >= 0) {
        d = pixel_ray(cam, px, py);
        const float ba = A.bary[2 * pix], bb = A.bary[2 * pix + 1];
        const float bc = 1.f - ba - bb;
        const int3 id = A.faces[f];
        vid[0] = id.x;
        vid[1] = id.y;
        vid[2] = id.z;
        bw[0] = ba;
        bw[1] = bb;
        bw[2] = bc;
        const float* P = A.verts + (long long)b * A.N * 3;
        v0 = ld3(P + 3 * id.x);
        v1 = ld3(P + 3 * id.y);
        v2 = ld3(P + 3 * id.z);
        const float* VN = A.vnormal + (long long)view * A.N * 3;
        const float3 n0 = ld3(VN + 3 * id.x), n1 = ld3(VN + 3 * id.y), n2 = ld3(VN + 3 * id.z);
        if (A.l1_state) {  // d L1 / d render (k_l1_grad's arithmetic)
            G = make_float3(0.f, 0.f, 0.f);
            if (!A.l1_mask || A.l1_mask[pix]) {
                const float3 r = ld3(A.l1_render + 3 * pix);
                float3 t;
                if (tma) {  // this tile's target is in shared memory already (the centre tap)
                    const float4 c = s_tgt[(py - ty0 + A.ifs) * e_st + (px - tx0 + A.ifs)];
                    t = make_float3(c.x, c.y, c.z);
                } else {
                    t = ld3(A.target + 3 * pix);
                }
                G = make_float3(l1_grad(l1_diff(r.x, t.x), l1_scale), l1_grad(l1_diff(r.y, t.y), l1_scale),
                                l1_grad(l1_diff(r.z, t.z), l1_scale));
            }
        } else {
            G = ld3(A.grad + 3 * pix);
        }
        frag = ba * v0 + bb * v1 + bc * v2;
        const float3 pnu = ba * n0 + bb * n1 + bc * n2;
        const float pnv = sqrtf(pnu.x * pnu.x + pnu.y * pnu.y + pnu.z * pnu.z);
        float3 pn = pnu / pnv;
        bool flipped = false;
        if (dot(pn, d) > 0.f) {
            pn = -pn;
            flipped = true;
        }
        const float* sh = A.sh + (long long)view * 27;
        float3 alb = make_float3(0.f, 0.f, 0.f);
        float3 coal = make_float3(1.f, 1.f, 1.f);
        if constexpr (SHADED) coal = sh_illum(sh, pn);
        gA = G * coal;  // d loss / d albedo
        const float* tcp = A.texcoords + (long long)f * 6;
        if constexpr (vcol) {
            const float* Cc = A.colors + (long long)b * A.N * 3;
            const float3 c0 = ld3(Cc + 3 * id.x), c1 = ld3(Cc + 3 * id.y), c2 = ld3(Cc + 3 * id.z);
            alb = ba * c0 + bb * c1 + bc * c2;
            gbc = make_float3(dot(gA, c0), dot(gA, c1), dot(gA, c2));
        } else if constexpr (bilinear) {
            // bilinear sampling: texture gradient to the four texels, and the
            // exact derivative of the sample w.r.t. the texel position
            const float2 t0 = make_float2(tcp[0], 1.f - tcp[1]);
            const float2 t1 = make_float2(tcp[2], 1.f - tcp[3]);
            const float2 t2 = make_float2(tcp[4], 1.f - tcp[5]);
            const float2 uv = t0 * ba + t1 * bb + t2 * bc;
            const BilinearTaps tp = bilinear_taps(uv.x * A.tex_w, uv.y * A.tex_h, A.tex_w, A.tex_h);
            const float* T = A.texture + (long long)b * A.tex_h * A.tex_w * 3;
            const float3 c00 = ld3(T + tp.o00), c10 = ld3(T + tp.o10), c01 = ld3(T + tp.o01), c11 = ld3(T + tp.o11);
            const float w00 = (1.f - tp.fx) * (1.f - tp.fy), w10 = tp.fx * (1.f - tp.fy),
                        w01 = (1.f - tp.fx) * tp.fy, w11 = tp.fx * tp.fy;
            alb = c00 * w00 + c10 * w10 + c01 * w01 + c11 * w11;
            float* tg = A.tex_grad + (long long)b * A.tex_h * A.tex_w * 3;
            const long long off[4] = {tp.o00, tp.o10, tp.o01, tp.o11};
            const float wt[4] = {w00, w10, w01, w11};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                atomicAdd(tg + off[q] + 0, gA.x * wt[q]);
                atomicAdd(tg + off[q] + 1, gA.y * wt[q]);
                atomicAdd(tg + off[q] + 2, gA.z * wt[q]);
            }
            const float3 dx = (c10 - c00) * (1.f - tp.fy) + (c11 - c01) * tp.fy;
            const float3 dy = (c01 - c00) * (1.f - tp.fx) + (c11 - c10) * tp.fx;
            const float gu = dot(gA, dx) * A.tex_w, gv = dot(gA, dy) * A.tex_h;
            gbc = make_float3(gu * t0.x + gv * t0.y, gu * t1.x + gv * t1.y, gu * t2.x + gv * t2.y);
        } else if constexpr (textured) {
            const float2 t0 = make_float2(tcp[0], 1.f - tcp[1]);
            const float2 t1 = make_float2(tcp[2], 1.f - tcp[3]);
            const float2 t2 = make_float2(tcp[4], 1.f - tcp[5]);
            float2 uv = t0 * ba + t1 * bb + t2 * bc;
            uv.x = uv.x * A.tex_w;
            uv.y = uv.y * A.tex_h;
            uv.x = fminf(fmaxf(uv.x, 0.f), (float)(A.tex_w - 1));
            uv.y = fminf(fmaxf(uv.y, 0.f), (float)(A.tex_h - 1));
            const float LU = (int)(uv.x - 0.5f) + 0.5f, HU = (int)(uv.x - 0.5f) + 1.5f;
            const float LV = (int)(uv.y - 0.5f) + 0.5f, HV = (int)(uv.y - 0.5f) + 1.5f;
            const float* T = A.texture + (long long)b * A.tex_h * A.tex_w * 3;
            const float3 cLL = ld3(T + 3LL * A.tex_w * (int)LV + 3 * (int)LU);
            const float3 cLH = ld3(T + 3LL * A.tex_w * (int)HV + 3 * (int)LU);
            const float3 cHL = ld3(T + 3LL * A.tex_w * (int)LV + 3 * (int)HU);
            const float3 cHH = ld3(T + 3LL * A.tex_w * (int)HV + 3 * (int)HU);
            // the reference's bilinear albedo used for the SH terms
            // (CUDABasedRasterizationGrad.cu:242-243), weight pairs as written there
            alb = (uv.y - LV) * (((uv.x - LU) * cLL) + ((HU - uv.x) * cHL)) +
                  (HV - uv.y) * (((uv.x - LU) * cLH) + ((HU - uv.x) * cHH));
            if (!flipped) {
                float* tg = A.tex_grad + (long long)b * A.tex_h * A.tex_w * 3 + 3LL * ((int)LV * A.tex_w + (int)LU);
                atomicAdd(tg + 0, gA.x);
                atomicAdd(tg + 1, gA.y);
                atomicAdd(tg + 2, gA.z);
            }
            float3 du, dv;
            image_gradient(T, uv.x, uv.y, A.tex_w, A.tex_h, A.tfs, du, dv);
            const float gu = dot(gA, du), gv = dot(gA, dv);
            gbc = make_float3(gu * (t0.x * A.tex_w) + gv * (t0.y * A.tex_h), gu * (t1.x * A.tex_w) + gv * (t1.y * A.tex_h),
                              gu * (t2.x * A.tex_w) + gv * (t2.y * A.tex_h));
        }
        if constexpr (SHADED) {
            // SH coefficients: G_r * albedo_r * basis(pn)
            const float basis[9] = {1.f, pn.y, pn.z, pn.x, pn.x * pn.y, pn.z * pn.y, 3.f * pn.z * pn.z - 1.f,
                                    pn.x * pn.z, pn.x * pn.x - pn.y * pn.y};
            const float gl[3] = {G.x * alb.x, G.y * alb.y, G.z * alb.z};
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 9; ++k) shg[9 * c + k] = gl[c] * basis[k];
            // d light / d normal (RendererUtil.h:371-391), then the normalisation Jacobian
            float3 gno = make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float* s = sh + 9 * c;
                const float3 row = make_float3(s[3] + s[4] * pn.y + s[7] * pn.z + s[8] * 2.f * pn.x,
                                               s[1] + s[4] * pn.x + s[5] * pn.z + s[8] * -2.f * pn.y,
                                               s[2] + s[5] * pn.y + s[6] * 6.f * pn.z + s[7] * pn.x);
                gno += gl[c] * row;
            }
            const float v2n = pnv * pnv, v3n = v2n * pnv;
            const float gu = dot(gno, pnu);
            gnu = (gno * v2n - pnu * gu) / v3n;
            gbc += make_float3(dot(gnu, n0), dot(gnu, n1), dot(gnu, n2));
        }
    }
    if (!tma) {  // (TMA mode: the tile's target was spread before its pixel work)
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this tile's copies (the next tile's stay in flight)
        __syncthreads();
    }
    if (f >= 0) {
        // model -> data: -G^T dTarget/d(u,v) d(u,v)/d(frag) d(frag)/d(v)
        float3 m = make_float3(0.f, 0.f, 0.f);
        {
            const int fs = A.ifs;
            float gu = 0.f, gv = 0.f;
            if (px >= fs + 1 && py >= fs + 1 && px < W - (fs + 1) && py < H - (fs + 1)) {
                // taps weighted (x, y)/(x^2 + y^2), normalised by sum |x|/(x^2 + y^2)
                // (imageGradient, RendererUtil.h:566-620), contracted with G
                if (staged) {
                    const int e = BT + 2 * fs, ew = 2 * fs + 1;
                    const int s0 = (py - ty0) * e + (px - tx0);
                    switch (fs) {
                        case 1: taps_fs<1>(s_tgt, s0, G, gu, gv); break;
                        case 2: taps_fs<2>(s_tgt, s0, G, gu, gv); break;
                        case 3: taps_fs<3>(s_tgt, s0, G, gu, gv); break;
                        default:
                            for (int j = 0; j < ew; ++j)
                                for (int i = 0; i < ew; ++i) {
                                    const float2 w = s_tap[j * ew + i];
                                    const float4 I = s_tgt[s0 + j * e + i];
                                    const float gi = G.x * I.x + G.y * I.y + G.z * I.z;
                                    gu += gi * w.x;
                                    gv += gi * w.y;
                                }
                    }
                    gu /= s_norm;
                    gv /= s_norm;
                } else {
                    float norm = 0.f;
                    for (int j = -fs; j <= fs; ++j)
                        for (int i = -fs; i <= fs; ++i) {
                            const float den = (float)(i * i + j * j);
                            if (den == 0.f) continue;
                            const float3 I = ld3(tgt + 3 * ((long long)(py + j) * W + (px + i)));
                            const float gi = dot(G, I);
                            gu += gi * ((float)i / den);
                            gv += gi * ((float)j / den);
                            norm += fabsf((float)i / den);
                        }
                    gu /= norm;
                    gv /= norm;
                }
            }
            if (gu != 0.f || gv != 0.f) {
                // pixel position of the fragment, P = K (E frag), and its
                // Jacobian d(u, v)/d frag = (KE_0 - u KE_2, KE_1 - v KE_2) / P_z
                const float* KE = cam.KE;
                const float3 Pp = make_float3(KE[0] * frag.x + KE[1] * frag.y + KE[2] * frag.z + cam.Kt[0],
                                              KE[3] * frag.x + KE[4] * frag.y + KE[5] * frag.z + cam.Kt[1],
                                              KE[6] * frag.x + KE[7] * frag.y + KE[8] * frag.z + cam.Kt[2]);
                if (fabsf(Pp.z) > 0.0001f) {
                    const float iz = 1.f / Pp.z;
                    const float dx = -Pp.x * iz * iz, dy = -Pp.y * iz * iz;
                    m.x = -(gu * (iz * KE[0] + dx * KE[6]) + gv * (iz * KE[3] + dy * KE[6]));
                    m.y = -(gu * (iz * KE[1] + dx * KE[7]) + gv * (iz * KE[4] + dy * KE[7]));
                    m.z = -(gu * (iz * KE[2] + dx * KE[8]) + gv * (iz * KE[5] + dy * KE[8]));
                }
            }
        }
        // data -> model through the barycentric Jacobian
        if constexpr (PARITY) {
            const float3 o = make_float3(cam.ro[0], cam.ro[1], cam.ro[2]);
            bary_jacobian_apply(o, d, v0, v1, v2, gbc, gp);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                gp[3 * i + 0] += m.x * bw[i];
                gp[3 * i + 1] += m.y * bw[i];
                gp[3 * i + 2] += m.z * bw[i];
            }
        } else {
            float3 r0, r1;
            float3 q = m;
            if (bary_rows(d, v0, v1, v2, r0, r1)) q += (gbc.x - gbc.z) * r0 + (gbc.y - gbc.z) * r1;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                gp[3 * i + 0] = q.x * bw[i];
                gp[3 * i + 1] = q.y * bw[i];
                gp[3 * i + 2] = q.z * bw[i];
            }
        }
    }
    // per-vertex contributions, merged inside the warp: lanes are matched by
    // face id (a face fixes all three vertices), and every 8th member of a
    // group (by lane order) sums its own row and the next 7 members' rows from
    // shared memory and issues one reduction per value and vertex.  The cap
    // bounds the loop (unrolled, its loads issue together) at the cost of a
    // second set of reductions for the rare group of more than 8 lanes.
    {
        float* row = s_red[warp][lane];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            row[NVV * i + 0] = gp[3 * i];
            row[NVV * i + 1] = gp[3 * i + 1];
            row[NVV * i + 2] = gp[3 * i + 2];
            row[NVV * i + 3] = gA.x * bw[i];
            row[NVV * i + 4] = gA.y * bw[i];
            row[NVV * i + 5] = gA.z * bw[i];
            if constexpr (SHADED) {
                row[NVV * i + 6] = gnu.x * bw[i];
                row[NVV * i + 7] = gnu.y * bw[i];
                row[NVV * i + 8] = gnu.z * bw[i];
            }
        }
        __syncwarp();
        const unsigned grp = __match_any_sync(0xffffffffu, f);
        const int rank = __popc(grp & ((1u << lane) - 1u));
        if (f >= 0 && rank % 8 == 0) {  // leader of up to 8 members: itself and the next 7
            float4 acc[NROW / 4];
#pragma unroll
            for (int k = 0; k < NROW / 4; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
            unsigned mm = grp & ~((1u << lane) - 1u);
            for (int q = 0; q < 8 && mm; ++q, mm &= mm - 1) {
                const float4* r = reinterpret_cast<const float4*>(s_red[warp][__ffs(mm) - 1]);
#pragma unroll
                for (int k = 0; k < NROW / 4; ++k) {
                    const float4 x = r[k];
                    acc[k].x += x.x;
                    acc[k].y += x.y;
                    acc[k].z += x.z;
                    acc[k].w += x.w;
                }
            }
            const float* a = reinterpret_cast<const float*>(acc);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const long long o3 = ((long long)b * A.N + vid[i]) * 3;
                atomicAdd(A.vpos_grad + o3 + 0, a[NVV * i + 0]);
                atomicAdd(A.vpos_grad + o3 + 1, a[NVV * i + 1]);
                atomicAdd(A.vpos_grad + o3 + 2, a[NVV * i + 2]);
                if constexpr (vcol) {
                    atomicAdd(A.vcol_grad + o3 + 0, a[NVV * i + 3]);
                    atomicAdd(A.vcol_grad + o3 + 1, a[NVV * i + 4]);
                    atomicAdd(A.vcol_grad + o3 + 2, a[NVV * i + 5]);
                }
                if constexpr (SHADED) {
                    atomicAdd(A.nrm_grad + o3 + 0, a[NVV * i + 6]);
                    atomicAdd(A.nrm_grad + o3 + 1, a[NVV * i + 7]);
                    atomicAdd(A.nrm_grad + o3 + 2, a[NVV * i + 8]);
                }
            }
        }
    }
    // SH: reduce over the CTA, one atomic per coefficient
    if constexpr (SHADED) {
#pragma unroll
        for (int k = 0; k < 27; ++k) {
            float v = shg[k];
#pragma unroll
            for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o2);
            if (lane == 0) s_sh[warp][k] = v;
        }
        __syncthreads();
        if (threadIdx.x < 27) {
            float v = 0.f;
            for (int w = 0; w < BNT / 32; ++w) v += s_sh[w][threadIdx.x];
            if (v != 0.f) atomicAdd(A.sh_grad + (long long)view * 27 + threadIdx.x, v);
        }
    }
    __syncthreads();  // the next iteration's prefetch reuses this tile's buffer
    if constexpr (DYN) g = s_claimed[(it + 1) & 1];
    else g += gridDim.x;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Normal chain, per (frame, vertex): for every incident face g = (x, y, z)
// with unnormalised normal N_g = (y - x) x (z - x), the gradient reaching N_g
// is the sum of the three vertex-normal gradients; d N_g / d vertex gives
//   x: g x (z - y),  y: (z - x) x g,  z: g x (y - x).
__global__ void k_normal_chain(int B, int N, const int3* __restrict__ faces, const int* __restrict__ vf,
                               const int2* __restrict__ vf_id, const float* __restrict__ verts,
                               const float* __restrict__ nrm_grad, float* __restrict__ vpos_grad) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * N) return;
    const int b = (int)(i / N), v = (int)(i % N);
    const float* P = verts + (long long)b * N * 3;
    const float* Gn = nrm_grad + (long long)b * N * 3;
    const int2 r = vf_id[v];
    float3 acc = make_float3(0.f, 0.f, 0.f);
    for (int k = r.x; k < r.x + r.y; ++k) {
        const int3 f = faces[vf[k]];
        const float3 g = ld3(Gn + 3 * f.x) + ld3(Gn + 3 * f.y) + ld3(Gn + 3 * f.z);
        const float3 x = ld3(P + 3 * f.x), y = ld3(P + 3 * f.y), z = ld3(P + 3 * f.z);
        if (v == f.x) acc += cross(g, z - y);
        else if (v == f.y) acc += cross(z - x, g);
        else acc += cross(g, y - x);
    }
    float* o = vpos_grad + i * 3;
    o[0] += acc.x;
    o[1] += acc.y;
    o[2] += acc.z;
}

}  // namespace

// CTAs of a persistent launch: as many as fit on the GPU at once (each walks
// tiles blockIdx.x, + gridDim.x, ...), never more than the tiles
template <class K>
static unsigned persistent_grid(K kernel, long long tiles) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, BNT, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    const long long g = (long long)sms * per_sm;
    return (unsigned)std::max<long long>(1, std::min(g, tiles));
}

hc_status raster_layout(RasterWorkspace& ws);

// The target image [V][H][W][3] as a 3-D tensor map {3W, H, V} (floats) with a
// box of kRawX x (16 + 2 ifs) x 1 for the adjoint's TMA staging.  False when
// the layout does not allow it (cameras of different sizes, rows that are not
// 16-byte multiples, an unaligned base, a filter wider than the staged tile,
// no driver entry point): the adjoint then stages with cp.async.
static bool target_tensor_map(const RasterWorkspace& ws, const float* target, int V, int ifs, CUtensorMap* map) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<Encode>(fn);
        cudaGetLastError();
    }
    if (!encode || ifs > MAXFS || ((uintptr_t)target & 15) != 0 || ws.cam_w.empty()) return false;
    const int W = ws.cam_w[0], H = ws.cam_h[0];
    for (size_t c = 1; c < ws.cam_w.size(); ++c)
        if (ws.cam_w[c] != W || ws.cam_h[c] != H) return false;
    if (W % 4 != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)3 * W, (cuuint64_t)H, (cuuint64_t)V};
    const cuuint64_t strides[2] = {(cuuint64_t)12 * W, (cuuint64_t)12 * W * H};
    const cuuint32_t box[3] = {(cuuint32_t)kRawX, (cuuint32_t)(BT + 2 * ifs), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(target), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

hc_status raster_backward(const Topology& topo, RasterWorkspace& ws, DevBuf& nrm_ws, cudaStream_t s, int B, int C,
                          int albedo, int shading, int ifs, int tfs, const float* grad,
                          const float* verts, const float* colors, const float* texture, int tex_h, int tex_w,
                          const float* sh, const float* target, const float* vnormal, const float* bary,
                          const int* face, const float* extr, const float* intr, float* vpos_grad,
                          float* vcol_grad, float* tex_grad, float* sh_grad, int parity, const L1Fuse* l1) {
    const int V = B * C, N = topo.N;
    HC_TRY(raster_layout(ws));
    HC_TRY(ws.cams.ensure(sizeof(ViewCam) * (size_t)std::max(V, ws.cap_views)));
    const bool shaded = shading == kShaded;
    if (shaded) HC_TRY(nrm_ws.ensure(sizeof(float) * 3 * (size_t)B * N));
    if (vpos_grad) HC_CUDA(cudaMemsetAsync(vpos_grad, 0, sizeof(float) * 3 * (size_t)B * N, s));
    if (vcol_grad) HC_CUDA(cudaMemsetAsync(vcol_grad, 0, sizeof(float) * 3 * (size_t)B * N, s));
    if (tex_grad && tex_h > 0 && tex_w > 0)
        HC_CUDA(cudaMemsetAsync(tex_grad, 0, sizeof(float) * 3 * (size_t)B * tex_h * tex_w, s));
    if (sh_grad) HC_CUDA(cudaMemsetAsync(sh_grad, 0, sizeof(float) * 27 * (size_t)V, s));
    if (shaded) HC_CUDA(cudaMemsetAsync(nrm_ws.ptr, 0, sizeof(float) * 3 * (size_t)B * N, s));
    ViewCam* cams = ws.cams.as<ViewCam>();
    k_view_setup<<<div_up(V, 64), 64, 0, s>>>(V, C, extr, intr, ws.layout.as<CamLayout>(), ws.P_frame, ws.T_frame,
                                              ws.Tb_frame, cams);
    HC_CHECK_LAUNCH();
    BwdArgs A;
    A.B = B;
    A.C = C;
    A.N = N;
    A.F = topo.F;
    A.Tb_frame = ws.Tb_frame;
    A.fd_frame = FastDiv((unsigned)ws.Tb_frame);
    A.fd_est = FastDiv((unsigned)(BT + 2 * ifs));
    A.tile_cam_b = ws.tile_cam_b.as<int>();
    A.albedo = albedo;
    A.shading = shading;
    A.ifs = ifs;
    A.tfs = tfs;
    A.tex_w = tex_w;
    A.tex_h = tex_h;
    A.faces = topo.faces.as<int3>();
    A.texcoords = topo.texcoords.as<float>();
    A.grad = grad;
    A.verts = verts;
    A.colors = colors;
    A.texture = texture;
    A.sh = sh;
    A.target = target;
    A.vnormal = vnormal;
    A.bary = bary;
    A.face = face;
    A.vpos_grad = vpos_grad;
    A.vcol_grad = vcol_grad;
    A.tex_grad = tex_grad;
    A.sh_grad = sh_grad;
    A.nrm_grad = shaded ? nrm_ws.as<float>() : nullptr;
    HC_TRY(ws.stats.ensure(sizeof(RasterStats)));
    A.err = &ws.stats.as<RasterStats>()->overflow;
    A.l1_state = l1 ? l1->state : nullptr;
    A.l1_render = l1 ? l1->render : nullptr;
    A.l1_mask = l1 ? l1->mask : nullptr;
    const long long tiles = (long long)B * ws.Tb_frame;
    HC_REQUIRE(tiles < (1ll << 31), "too many adjoint tiles in one call (%lld)", tiles);
    HC_TRY(ws.claim_b.ensure(sizeof(unsigned)));
    A.claim = ws.claim_b.as<unsigned>();
    const bool dyn = ws.adjoint_dynamic != 0;
    if (dyn) HC_CUDA(cudaMemsetAsync(A.claim, 0, sizeof(unsigned), s));
    // the target's tensor map for the TMA staging, where its layout allows it
    CUtensorMap tmap;
    memset(&tmap, 0, sizeof(tmap));
    const int use_tma = target_tensor_map(ws, target, V, ifs, &tmap) ? 1 : 0;
    ws.clock.begin(kKRenderGrad, s);
    const int alb = albedo == kVertexColor ? kAlbVcol
                    : albedo == kTextured ? kAlbTex
                    : albedo == kTexturedBilinear ? kAlbTexBilinear : kAlbNone;
    const int sel = (shaded ? 8 : 0) + alb * 2 + (parity ? 1 : 0);
    switch (sel) {
#define HC_GRAD_CASE(SH, AL, PA)                                                                              \
    case (SH ? 8 : 0) + AL * 2 + PA:                                                                          \
        if (dyn)                                                                                              \
            k_render_grad<SH, AL, PA, true><<<persistent_grid(k_render_grad<SH, AL, PA, true>, tiles), BNT, 0, s>>>( \
                A, cams, tiles, tmap, use_tma);                                                               \
        else                                                                                                  \
            k_render_grad<SH, AL, PA, false><<<persistent_grid(k_render_grad<SH, AL, PA, false>, tiles), BNT, 0, s>>>( \
                A, cams, tiles, tmap, use_tma);                                                               \
        break;
        HC_GRAD_CASE(false, kAlbVcol, false)
        HC_GRAD_CASE(false, kAlbVcol, true)
        HC_GRAD_CASE(false, kAlbTex, false)
        HC_GRAD_CASE(false, kAlbTex, true)
        HC_GRAD_CASE(false, kAlbNone, false)
        HC_GRAD_CASE(false, kAlbNone, true)
        HC_GRAD_CASE(true, kAlbVcol, false)
        HC_GRAD_CASE(true, kAlbVcol, true)
        HC_GRAD_CASE(true, kAlbTex, false)
        HC_GRAD_CASE(true, kAlbTex, true)
        HC_GRAD_CASE(true, kAlbNone, false)
        HC_GRAD_CASE(true, kAlbNone, true)
        HC_GRAD_CASE(false, kAlbTexBilinear, false)
        HC_GRAD_CASE(false, kAlbTexBilinear, true)
        HC_GRAD_CASE(true, kAlbTexBilinear, false)
        HC_GRAD_CASE(true, kAlbTexBilinear, true)
#undef HC_GRAD_CASE
    }
    HC_CHECK_LAUNCH();
    ws.clock.end(kKRenderGrad, s);
    if (shaded) {
        ws.clock.begin(kKNormalChain, s);
        k_normal_chain<<<div_up((long long)B * N, 256), 256, 0, s>>>(B, N, topo.faces.as<int3>(), topo.vf.as<int>(),
                                                                     topo.vf_id.as<int2>(), verts, nrm_ws.as<float>(),
                                                                     vpos_grad);
        HC_CHECK_LAUNCH();
        ws.clock.end(kKNormalChain, s);
    }
    return HC_OK;
}

}  // namespace hc
