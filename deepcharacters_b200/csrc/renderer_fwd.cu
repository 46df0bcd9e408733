// Forward rasterizer: camera set-up, vertex normals, triangle set-up with
// screen-tile binning, spill-over raster and the per-tile visibility resolve
// fused with barycentric / face-id / albedo / SH shading output.
//
// Reference behaviour (CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cu):
// one thread per (view, triangle) loops over the triangle's pixel bbox twice,
// first an int atomicMin on the quantised depth, then a racy write of every
// triangle whose depth equals the minimum.  Here each pixel is owned by one
// thread of its tile's CTA: the triangles binned to the tile are staged in
// shared memory and every thread keeps the minimum (depth_q, triangle) of its
// pixel in registers, so the common path has no atomics and the winner among
// equal depths is deterministic (smallest triangle id).  Triangles beyond the
// tile's bin capacity go through a spill list resolved with a 64-bit packed
// atomicMin and merged afterwards.
#include <algorithm>

#include "renderer.cuh"

namespace hc {

// ---------------------------------------------------------------------------
// camera set-up: one thread per view (reference initializeCamerasDevice,
// CUDABasedRasterization.cu:23-67, which runs <<<1,1>>> per frame)
// ---------------------------------------------------------------------------
__global__ void k_view_setup(int V, int C, const float* __restrict__ extr, const float* __restrict__ intr,
                             const CamLayout* __restrict__ layout, long long P_frame, long long T_frame,
                             long long Tb_frame, ViewCam* __restrict__ cams) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    {
        const CamLayout L = layout[v % C];
        const long long b = v / C;
        ViewCam& c = cams[v];
        c.W = L.W;
        c.H = L.H;
        c.tiles_x = L.tiles_x;
        c.tiles_x_b = L.tiles_x_b;
        c.fd_tiles_x = L.fd_tiles_x;
        c.fd_tiles_x_b = L.fd_tiles_x_b;
        c.pix_base = b * P_frame + L.pix;
        c.tile_base = b * T_frame + L.tile;
        c.tile_base_b = b * Tb_frame + L.tile_b;
    }
    const float* e = extr + 12 * (long long)v;
    const float* k = intr + 9 * (long long)v;
    M44 E, K;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        E.e[i] = (i % 5 == 0) ? 1.f : 0.f;
        K.e[i] = (i % 5 == 0) ? 1.f : 0.f;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        K.e[4 * r + 0] = k[3 * r + 0];
        K.e[4 * r + 1] = k[3 * r + 1];
        K.e[4 * r + 2] = k[3 * r + 2];
        K.e[4 * r + 3] = 0.f;
        E.e[4 * r + 0] = e[4 * r + 0];
        E.e[4 * r + 1] = e[4 * r + 1];
        E.e[4 * r + 2] = e[4 * r + 2];
        E.e[4 * r + 3] = e[4 * r + 3];
    }
    const M44 invE = inverse44(E);
    const M44 invP = inverse44(mul44(K, E));
    ViewCam& c = cams[v];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        c.invP[i] = invP.e[i];
        c.invE[i] = invE.e[i];
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) c.ext[i] = e[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) c.intr[i] = k[i];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
            c.KE[3 * r + cc] = k[3 * r + 0] * e[cc] + k[3 * r + 1] * e[4 + cc] + k[3 * r + 2] * e[8 + cc];
        c.Kt[r] = k[3 * r + 0] * e[3] + k[3 * r + 1] * e[7] + k[3 * r + 2] * e[11];
    }
    // camera centre: last column of inv(E), dehomogenised
    float4 o = make_float4(invE.e[3], invE.e[7], invE.e[11], invE.e[15]);
    const float w = o.w;
    o.x /= w;
    o.y /= w;
    o.z /= w;
    c.ro[0] = o.x;
    c.ro[1] = o.y;
    c.ro[2] = o.z;
    c.ro_s[0] = o.x / 1000.f;
    c.ro_s[1] = o.y / 1000.f;
    c.ro_s[2] = o.z / 1000.f;
}

// ---------------------------------------------------------------------------
// vertex normals: unnormalised sum of incident face normals, in increasing
// face order (reference renderFaceNormalDevice / renderVertexNormalDevice,
// CUDABasedRasterization.cu:122-174, computed once per frame and written for
// every camera of the [B,C,N,3] output)
// ---------------------------------------------------------------------------
__global__ void k_vertex_normals(int B, int C, int N, const int3* __restrict__ faces,
                                 const int* __restrict__ vf, const int2* __restrict__ vf_id,
                                 const float* __restrict__ verts, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * N) return;
    const int b = (int)(i / N);
    const int v = (int)(i % N);
    const float* P = verts + (long long)b * N * 3;
    const int2 r = vf_id[v];
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int k = r.x; k < r.x + r.y; ++k) {
        const int3 f = faces[vf[k]];
        const float3 v0 = ld3(P + 3 * f.x), v1 = ld3(P + 3 * f.y), v2 = ld3(P + 3 * f.z);
        const float3 fn = cross(v1 - v0, v2 - v0);
        if (k == r.x) {
            s = fn;
        } else {
            s.x = s.x + fn.x;
            s.y = s.y + fn.y;
            s.z = s.z + fn.z;
        }
    }
    for (int c = 0; c < C; ++c) st3(out + (((long long)b * C + c) * N + v) * 3, s);
}

// ---------------------------------------------------------------------------
// per-frame triangle constants
// ---------------------------------------------------------------------------
__global__ void k_tri_frame(int B, int F, int N, const int3* __restrict__ faces,
                            const float* __restrict__ verts, TriFrame* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)B * F) return;
    const int b = (int)(i / F);
    const int f = (int)(i % F);
    const float* P = verts + (long long)b * N * 3;
    const int3 id = faces[f];
    const float3 s0 = ld3(P + 3 * id.x) / 1000.f;
    const float3 s1 = ld3(P + 3 * id.y) / 1000.f;
    const float3 s2 = ld3(P + 3 * id.z) / 1000.f;
    const float3 n = cross(s1 - s0, s2 - s0);
    TriFrame t;
    t.a = make_float4(s0.x, s0.y, s0.z, n.x);
    t.b = make_float4(s1.x, s1.y, s1.z, n.y);
    t.c = make_float4(s2.x, s2.y, s2.z, n.z);
    out[i] = t;
}

// ---------------------------------------------------------------------------
// per-view vertex projection (reference projectVerticesDevice,
// CUDABasedRasterization.cu:98-115): once per (view, vertex) instead of three
// times per (view, triangle); the same function, so the same values
// ---------------------------------------------------------------------------
__global__ void k_project_vertices(int V, int C, int N, const float* __restrict__ verts,
                                   const ViewCam* __restrict__ cams, float4* __restrict__ proj) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)V * N) return;
    const int view = (int)(i / N), v = (int)(i % N);
    const ViewCam& cam = cams[view];
    const float3 p = project_point(cam.ext, cam.intr, ld3(verts + ((long long)(view / C) * N + v) * 3));
    proj[i] = make_float4(p.x, p.y, p.z, 0.f);
}

// ---------------------------------------------------------------------------
// per-view triangle set-up and screen-tile binning
//
// The pixel bbox is the reference's projectFacesDevice (CUDABasedRasterization.cu:
// 184-208): projected vertex extent +-0.5 px, clamped to the image, truncated to
// int.  Each (view, triangle) appends itself to every tile its bbox touches
// and its footprint reaches, taking a slot with one atomicAdd on the tile's
// counter; entries beyond the tile's capacity go to the spill list.
// ---------------------------------------------------------------------------
constexpr int kBinSmall = 9;  // tiles a thread bins on its own (a 3x3 box of tiles)

// Where a (tile, triangle) pair goes once it has a slot in the tile's bin:
// the bin itself, or beyond the bin's capacity the spill list (the first
// overflowing pair of a tile claims and clears the tile's spill key block).
struct BinSink {
    int TS, cap;
    int2* tile_state;
    int* bins;
    int2* spill;  // (tile of the call, triangle)
    long long spill_cap;
    unsigned long long* spill_keys;
    int spill_tile_cap;
    RasterStats* stats;

    __device__ __forceinline__ int place(int slot, long long key, int view, int local_tile, int f) const {
        if (slot < cap) {
            bins[key * cap + slot] = f;
            return 1;
        }
        if (slot == cap) {
            const int ks = atomicAdd(&stats->spill_tiles, 1);
            if (ks < spill_tile_cap) {
                unsigned long long* kp = spill_keys + (long long)ks * TS * TS;
                for (int p = 0; p < TS * TS; ++p) kp[p] = ~0ull;
                tile_state[key].y = ks + 1;
            } else {
                atomicOr(&stats->overflow, 2);
            }
        }
        const unsigned long long si = atomicAdd(&stats->spilled, 1ull);
        if ((long long)si < spill_cap) {
            spill[si] = make_int2((int)key, f);
        } else {
            atomicOr(&stats->overflow, 1);
        }
        return 0;
    }
};

__global__ void __launch_bounds__(256, 6) k_bin(int V, int C, int F, int N, int TS, int ts_shift, int cap,
                      const int3* __restrict__ faces, const float4* __restrict__ proj,
                      const ViewCam* __restrict__ cams, const TriFrame* __restrict__ tri_frame,
                      TriView* __restrict__ tri_view, int2* __restrict__ tile_state, int* __restrict__ bins,
                      int2* __restrict__ spill, long long spill_cap, unsigned long long* __restrict__ spill_keys,
                      int spill_tile_cap, RasterStats* __restrict__ stats) {
    // grid (triangle blocks, views): no 64-bit division per thread
    const int fi = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = fi < F;
    const int view = blockIdx.y;
    const long long i = (long long)view * F + fi;
    int f = 0;
    int x0 = 0, x1 = -1, y0 = 0, y1 = -1;
    // the view is the block's (grid y), so its image and tile grid are the same in every lane
    const ViewCam& cam = cams[view];
    const int W = cam.W, H = cam.H, tiles_x = cam.tiles_x;
    const long long tile_base = cam.tile_base;
    Footprint fp;
    if (live) {
        f = fi;
        const int b = view / C;
        const int3 id = faces[f];
        const float4* PV = proj + (long long)view * N;
        const float4 q0 = PV[id.x], q1 = PV[id.y], q2 = PV[id.z];
        const float3 p0 = make_float3(q0.x, q0.y, q0.z), p1 = make_float3(q1.x, q1.y, q1.z),
                     p2 = make_float3(q2.x, q2.y, q2.z);
        x0 = (int)fmaxf(fminf(p0.x, fminf(p1.x, p2.x)) - 0.5f, 0.f);
        y0 = (int)fmaxf(fminf(p0.y, fminf(p1.y, p2.y)) - 0.5f, 0.f);
        x1 = (int)fminf(fmaxf(p0.x, fmaxf(p1.x, p2.x)) + 0.5f, (float)(W - 1));
        y1 = (int)fminf(fmaxf(p0.y, fmaxf(p1.y, p2.y)) + 0.5f, (float)(H - 1));
        const TriS T = tri_from(tri_frame[(long long)b * F + f]);
        const float3 ro_s = make_float3(cam.ro_s[0], cam.ro_s[1], cam.ro_s[2]);
        TriView tv;
        tv.num = dot(T.s0, T.n) - dot(ro_s, T.n);
        // x1/y1 can be negative for triangles left of / above the image
        // (empty bbox); store them clamped to -1 so the 16-bit packing keeps
        // the bbox empty.
        // x0/y0 beyond the image also mean an empty bbox (x1 <= W-1); clamp
        // them to W/H so they fit the 16-bit field.
        const int cx1 = max(x1, -1), cy1 = max(y1, -1);
        const int cx0 = min(x0, W), cy0 = min(y0, H);
        tv.x01 = (cx0 & 0xffff) | (cx1 << 16);
        tv.y01 = (cy0 & 0xffff) | (cy1 << 16);
        // front-facing: the plane normal points towards the camera (num < 0)
        tv.dqmin = depth_lower_bound(tv.num, T.n, T, ro_s) | (tv.num < 0.f ? 0 : (int)0x80000000);
        fp = footprint(p0, p1, p2);
        // the tile resolve stages this record as it is (no vertex gathers there)
        tv.e01 = make_float4(fp.a[0], fp.b[0], fp.a[1], fp.b[1]);
        tv.e2c = make_float4(fp.a[2], fp.b[2], fp.c[0], fp.c[1]);
        tv.e2o = make_float4(fp.c[2], 0.f, 0.f, 0.f);
        tri_view[i] = tv;
    }
    const bool nonempty = live && x1 >= x0 && y1 >= y0;
    int tx0 = 0, tx1 = -1, ty0 = 0, ty1 = -1;
    if (nonempty) {
        tx0 = x0 >> ts_shift;  // TS = 2^ts_shift; the box is non-empty, so x0 <= x1 are >= 0
        tx1 = x1 >> ts_shift;
        ty0 = y0 >> ts_shift;
        ty1 = y1 >> ts_shift;
    }
    const int ntx = tx1 - tx0 + 1;
    const int nt = nonempty ? ntx * (ty1 - ty0 + 1) : 0;
    const bool big = nt > kBinSmall;
    BinSink sink{TS, cap, tile_state, bins, spill, spill_cap, spill_keys, spill_tile_cap, stats};
    unsigned long long nbinned = 0;
    const unsigned lane = threadIdx.x & 31;
    // boxes of up to kBinSmall tiles: each lane walks its own box
    const int my_nt = big ? 0 : nt;
    int cx = 0, cy = 0;  // column / row of tile k in the box, stepped without a division
    for (int k = 0; k < my_nt; ++k) {
        const int tx = tx0 + cx, ty = ty0 + cy;
        if (++cx == ntx) {
            cx = 0;
            ++cy;
        }
        // tiles of the box that the triangle's footprint misses get no entry
        if (nt > 1 && !footprint_overlaps(fp, max(tx * TS, x0), min(tx * TS + TS - 1, x1), max(ty * TS, y0),
                                          min(ty * TS + TS - 1, y1)))
            continue;
        const long long key = tile_base + ty * tiles_x + tx;
        nbinned += sink.place(atomicAdd(&tile_state[key].x, 1), key, view, (int)(key - tile_base), f);
    }
    // larger boxes: the warp takes them one at a time, a tile per lane
    unsigned pending = __ballot_sync(0xffffffffu, big);
    while (pending) {
        const int src = __ffs(pending) - 1;
        pending &= pending - 1;
        const int qv = view, qf = __shfl_sync(0xffffffffu, f, src);
        const int qtiles_x = tiles_x;
        const long long qbase = tile_base;
        const int qx0 = __shfl_sync(0xffffffffu, x0, src), qx1 = __shfl_sync(0xffffffffu, x1, src);
        const int qy0 = __shfl_sync(0xffffffffu, y0, src), qy1 = __shfl_sync(0xffffffffu, y1, src);
        Footprint qfp;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            qfp.a[e] = __shfl_sync(0xffffffffu, fp.a[e], src);
            qfp.b[e] = __shfl_sync(0xffffffffu, fp.b[e], src);
            qfp.c[e] = __shfl_sync(0xffffffffu, fp.c[e], src);
        }
        const int qtx0 = qx0 >> ts_shift, qty0 = qy0 >> ts_shift, qntx = (qx1 >> ts_shift) - qtx0 + 1;
        const int qnt = qntx * ((qy1 >> ts_shift) - qty0 + 1);
        // lane's tile k = lane + 32 j at (row cr, column cc), stepped by 32.
        // floor(a / n) for a <= 32, n <= 4096 from one reciprocal: (a + 1/2) / n
        // is at least 1/(2n) from an integer, far above the float error
        const float rq = 1.f / (float)qntx;
        const int step_r = (int)(32.5f * rq), step_c = 32 - step_r * qntx;
        int cr = (int)(((float)lane + 0.5f) * rq), cc = (int)lane - cr * qntx;
        for (int k = lane; k < qnt; k += 32) {
            const int tx = qtx0 + cc;
            const int ty = qty0 + cr;
            cc += step_c;
            cr += step_r;
            if (cc >= qntx) {
                cc -= qntx;
                ++cr;
            }
            if (!footprint_overlaps(qfp, max(tx * TS, qx0), min(tx * TS + TS - 1, qx1), max(ty * TS, qy0),
                                    min(ty * TS + TS - 1, qy1)))
                continue;
            const long long key = qbase + ty * qtiles_x + tx;
            nbinned += sink.place(atomicAdd(&tile_state[key].x, 1), key, qv, (int)(key - qbase), qf);
        }
    }
    // one counter update per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nbinned += __shfl_xor_sync(0xffffffffu, nbinned, o);
    if (lane == 0 && nbinned) atomicAdd(&stats->binned, nbinned);
}

__device__ __forceinline__ void unpack_bbox(const TriView& tv, int& x0, int& x1, int& y0, int& y1) {
    x0 = tv.x01 & 0xffff;
    x1 = tv.x01 >> 16;
    y0 = tv.y01 & 0xffff;
    y1 = tv.y01 >> 16;
}

// ---------------------------------------------------------------------------
// spill raster: (view, tile, triangle) items beyond the bin capacity, one
// thread each, 64-bit packed atomicMin per pixel of tile x bbox.  With
// `count_depth` set (diagnostics) the pass instead counts, per pixel, the
// spilled triangles that reach the final depth.
// ---------------------------------------------------------------------------
__global__ void k_spill(int C, int F, int TS, long long T_frame, const int* __restrict__ tile_cam,
                        const ViewCam* __restrict__ cams, const TriFrame* __restrict__ tri_frame,
                        const TriView* __restrict__ tri_view, const int2* __restrict__ tile_state,
                        const int2* __restrict__ spill, long long spill_cap, int spill_tile_cap,
                        unsigned long long* __restrict__ spill_keys, const RasterStats* __restrict__ stats,
                        const int* __restrict__ count_depth, int* __restrict__ tie_out) {
    // one warp per spilled (tile, triangle) entry, its lanes over the pixels
    // of the triangle's box in the tile (the per-pixel atomic minimum does
    // not depend on the order)
    const long long n = min((long long)stats->spilled, spill_cap);
    const int lane = threadIdx.x & 31;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
        const int2 it = spill[i];
        const long long g = it.x;
        const int f = it.y;
        const int view = (int)(g / T_frame) * C + tile_cam[g % T_frame];
        const ViewCam& cam = cams[view];
        const int tile = (int)(g - cam.tile_base);
        const int ks = tile_state[g].y - 1;
        if (ks < 0 || ks >= spill_tile_cap) continue;
        const int W = cam.W, H = cam.H, tiles_x = cam.tiles_x;
        const TriView tv = tri_view[(long long)view * F + f];
        const TriS Tr = tri_from(tri_frame[(long long)(view / C) * F + f]);
        const float3 ro_s = make_float3(cam.ro_s[0], cam.ro_s[1], cam.ro_s[2]);
        int x0, x1, y0, y1;
        unpack_bbox(tv, x0, x1, y0, y1);
        const int tx = tile % tiles_x, ty = tile / tiles_x;
        const int px0 = max(x0, tx * TS), px1 = min(x1, min(tx * TS + TS - 1, W - 1));
        const int py0 = max(y0, ty * TS), py1 = min(y1, min(ty * TS + TS - 1, H - 1));
        const int bw = px1 - px0 + 1, bh = py1 - py0 + 1;
        if (bw <= 0 || bh <= 0) continue;
        for (int q = lane; q < bw * bh; q += 32) {
            {
                const int px = px0 + q % bw, py = py0 + q / bw;
                const float3 dir = pixel_ray(cam, px, py);
                int dq;
                float a, b;
                if (!raster_hit(ro_s, dir, Tr, tv.num, dq, a, b)) continue;
                const int local = (py - ty * TS) * TS + (px - tx * TS);
                if (count_depth) {
                    const long long pix = cam.pix_base + (long long)py * W + px;
                    if (dq == count_depth[pix]) atomicAdd(&tie_out[pix], 1);
                } else {
                    const unsigned long long key = ((unsigned long long)(unsigned)dq << 32) | (unsigned)f;
                    atomicMin(&spill_keys[(long long)ks * TS * TS + local], key);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// tile resolve + shading
// ---------------------------------------------------------------------------
struct ShadeArgs {
    int B, C, N, F;
    const float4* proj;  // [V,N] projected vertices
    int albedo, shading;
    const int3* faces;
    const float* texcoords;
    const float* verts;
    const float* colors;
    const float* texture;
    int tex_w, tex_h;
    const float* sh;
    const float* vnormal;  // [B,C,N,3]
    float* bary;
    int* face;
    float* render;
    int* depth_q;
    int* tie_count;
    // fused image L1 (NULL sums: not fused)
    const float* l1_target;
    const unsigned char* l1_mask;
    float* l1_sum;     // [tiles * warps per tile]
    unsigned* l1_cnt;  // [tiles * warps per tile]
};

// colour of a pixel hit by face f at barycentrics (a, bb)
__device__ __forceinline__ float3 shade_pixel(const ShadeArgs& A, const ViewCam& cam, int view, int b, int f,
                                              float a, float bb, float3 dir) {
    const int3 id = A.faces[f];
    // the interpolated normal, only where the albedo or the shading reads it
    float3 pn = make_float3(0.f, 0.f, 0.f);
    if (A.albedo == kNormal || A.albedo == kLighting || A.shading == kShaded) {
        const float* VN = A.vnormal + ((long long)view * A.N) * 3;
        const float3 n0 = ld3(VN + 3 * id.x), n1 = ld3(VN + 3 * id.y), n2 = ld3(VN + 3 * id.z);
        pn = n0 * a + n1 * bb + n2 * (1.f - a - bb);
        pn = pn / length3(pn);
        if (dot(pn, dir) > 0.f) pn = -pn;
    }
    float3 color = make_float3(0.f, 0.f, 0.f);
    switch (A.albedo) {
        case kTextured: {
            const float* tc = A.texcoords + (long long)f * 6;
            const float2 t0 = make_float2(tc[0], 1.f - tc[1]);
            const float2 t1 = make_float2(tc[2], 1.f - tc[3]);
            const float2 t2 = make_float2(tc[4], 1.f - tc[5]);
            float2 uv = t0 * a + t1 * bb + t2 * (1.f - a - bb);
            uv.x = uv.x * A.tex_w;
            uv.y = uv.y * A.tex_h;
            uv.x = fmaxf(uv.x, 0.f);
            uv.x = fminf(uv.x, (float)(A.tex_w - 1));
            uv.y = fmaxf(uv.y, 0.f);
            uv.y = fminf(uv.y, (float)(A.tex_h - 1));
            const int lu = (int)(uv.x - 0.5f);
            const int lv = (int)(uv.y - 0.5f);
            const float* T = A.texture + (long long)b * A.tex_h * A.tex_w * 3;
            color = ld3(T + 3LL * A.tex_w * lv + 3 * lu);
            break;
        }
        case kTexturedBilinear: {
            const float* tc = A.texcoords + (long long)f * 6;
            const float2 t0 = make_float2(tc[0], 1.f - tc[1]);
            const float2 t1 = make_float2(tc[2], 1.f - tc[3]);
            const float2 t2 = make_float2(tc[4], 1.f - tc[5]);
            const float2 uv = t0 * a + t1 * bb + t2 * (1.f - a - bb);
            const float* T = A.texture + (long long)b * A.tex_h * A.tex_w * 3;
            color = bilinear_sample(T, bilinear_taps(uv.x * A.tex_w, uv.y * A.tex_h, A.tex_w, A.tex_h));
            break;
        }
        case kVertexColor: {
            const float* Cc = A.colors + (long long)b * A.N * 3;
            const float3 c0 = ld3(Cc + 3 * id.x), c1 = ld3(Cc + 3 * id.y), c2 = ld3(Cc + 3 * id.z);
            color = make_float3(c0.x * a + c1.x * bb + c2.x * (1.f - a - bb),
                                c0.y * a + c1.y * bb + c2.y * (1.f - a - bb),
                                c0.z * a + c1.z * bb + c2.z * (1.f - a - bb));
            break;
        }
        case kNormal:
            color = make_float3((1.f + pn.x) / 2.f, (1.f + pn.y) / 2.f, (1.f + pn.z) / 2.f);
            break;
        case kLighting:
        case kForegroundMask:
            color = make_float3(1.f, 1.f, 1.f);
            break;
        case kPosition:
        case kDepth: {
            const float* P = A.verts + (long long)b * A.N * 3;
            const float3 p0 = ld3(P + 3 * id.x), p1 = ld3(P + 3 * id.y), p2 = ld3(P + 3 * id.z);
            const float3 pos = make_float3(p0.x * a + p1.x * bb + p2.x * (1.f - a - bb),
                                           p0.y * a + p1.y * bb + p2.y * (1.f - a - bb),
                                           p0.z * a + p1.z * bb + p2.z * (1.f - a - bb));
            if (A.albedo == kPosition) {
                color = pos;
            } else {
                const float3 o = make_float3(cam.ro[0], cam.ro[1], cam.ro[2]);
                const float d = length3(o - pos);
                color = make_float3(d, d, d);
            }
            break;
        }
        case kUV: {
            const float* tc = A.texcoords + (long long)f * 6;
            const float2 t0 = make_float2(tc[0], 1.f - tc[1]);
            const float2 t1 = make_float2(tc[2], 1.f - tc[3]);
            const float2 t2 = make_float2(tc[4], 1.f - tc[5]);
            float2 uv = t0 * a + t1 * bb + t2 * (1.f - a - bb);
            uv.x = fminf(fmaxf(uv.x, 0.f), 1.f);
            uv.y = fminf(fmaxf(uv.y, 0.f), 1.f);
            color = make_float3(uv.x, uv.y, 0.f);
            break;
        }
        default:
            break;
    }
    if ((A.shading == kShaded && A.albedo != kNormal) || A.albedo == kLighting) {
        const float3 L = sh_illum(A.sh + (long long)view * 27, pn);
        color = make_float3(L.x * color.x, L.y * color.y, L.z * color.z);
    }
    return color;
}

struct TileTri {
    int4 hdr;        // column mask, row mask (tile-relative bbox), depth lower bound, face id
    float4 ea;       // footprint edges 0, 1: (a0, b0, a1, b1)
    float4 nm;       // ray-plane numerator, footprint offsets c0, c1, c2
    float4 eb;       // footprint edge 2: (a2, b2, -, -)
    float4 a, b, c;  // TriFrame
};

// Hit test with an early depth rejection: the quantised depth int(t * 1e4) is
// known as soon as t is, so a triangle that cannot reach the pixel's current
// best depth skips the edge tests.  Accepted hits and their depth / barycentrics
// are those of raster_hit.
__device__ __forceinline__ bool raster_hit_below(float3 ro_s, float3 dir, const TriS& T, float num,
                                                 unsigned best_d, int& depth_q, float& a, float& b) {
    const float ndr = dot(dir, T.n);
    if (fabsf(ndr) < 0.0000001f) return false;
    const float t = num / ndr;
    if (t < 0.f) return false;
    depth_q = (int)(t * 10000.f);
    if ((unsigned)depth_q > best_d) return false;
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
    return (a >= -0.001f) && (b >= -0.001f) && (a <= 1.001f) && (b <= 1.001f);
}

// bits lo..hi of a 32-bit mask (empty when hi < lo)
__device__ __forceinline__ unsigned bit_range(int lo, int hi) {
    return hi < lo ? 0u : ((2u << hi) - 1u) & ~((1u << lo) - 1u);
}

// TIES: the call asked for the per-pixel count of hits at the winning depth
// (diagnostics); without it the count is compiled out, which frees a register
// of the scan and shortens its updates
template <int TS, bool TIES>
__global__ void __launch_bounds__(TS* TS, TS == 8 ? 20 : (TS == 16 ? 5 : 1)) k_resolve(ShadeArgs A, FastDiv fd_frame,
                                                   const int* __restrict__ tile_cam, int cap,
                                                   const ViewCam* __restrict__ cams,
                                                   const TriFrame* __restrict__ tri_frame,
                                                   const TriView* __restrict__ tri_view,
                                                   const int2* __restrict__ tile_state,
                                                   const int* __restrict__ bins,
                                                   const unsigned long long* __restrict__ spill_keys,
                                                   int spill_tile_cap, long long n_tiles,
                                                   unsigned long long* __restrict__ claim) {
    constexpr int NT = TS * TS;
    constexpr int CHUNK = NT > 256 ? 256 : NT;  // triangles staged per round
    constexpr int SB = CHUNK == 64 ? 6 : 8;     // slot bits of a sort key
    constexpr unsigned kNoKey = 0xffffffffu;
    __shared__ TileTri s_tri[CHUNK];             // staged triangles in key order
    __shared__ unsigned s_key[CHUNK];            // per warp: its keys, sorted
    __shared__ unsigned char s_rank[CHUNK];       // position of each slot in key order
    // Resident CTAs claim the tiles of the call from a counter (the frame's
    // cameras concatenated), kClaim consecutive tiles per atomic: no launch
    // cost per tile, tiles of very different cost still balance, and the one
    // counter sees a quarter of the atomics.  Thread 0 claims into the slot of
    // this claim's parity; the slot is rewritten two claims later, after every
    // thread has passed the next claim's barrier.
    constexpr int kClaim = 4;
    __shared__ long long s_g[2];
    for (int it = 0;; ++it) {
    if (it % kClaim == 0) {
        if (threadIdx.x == 0) s_g[(it / kClaim) & 1] = (long long)atomicAdd(claim, (unsigned long long)kClaim);
        __syncthreads();
    }
    const long long g = s_g[(it / kClaim) & 1] + it % kClaim;
    if (g >= n_tiles) break;
    // tile -> (frame, camera, tile of the camera): the call has < 2^31 tiles
    const int b = (int)fd_frame.div((unsigned)g);
    const int view = b * A.C + tile_cam[fd_frame.mod((unsigned)g, (unsigned)b)];
    const ViewCam& cam = cams[view];
    const int tile = (int)(g - cam.tile_base);
    const int W = cam.W, H = cam.H;
    const int ty = (int)cam.fd_tiles_x.div((unsigned)tile), tx = (int)cam.fd_tiles_x.mod((unsigned)tile, ty);
    const int lx = threadIdx.x % TS, ly = threadIdx.x / TS;
    const int px = tx * TS + lx, py = ty * TS + ly;
    const unsigned col_bit = 1u << lx, row_bit = 1u << ly;
    const float cx = px + 0.5f, cy = py + 0.5f;
    const bool valid = px < W && py < H;
    const float3 ro_s = make_float3(cam.ro_s[0], cam.ro_s[1], cam.ro_s[2]);
    const float3 dir = pixel_ray(cam, px, py);
    const int2 st = tile_state[g];
    const int n = min(st.x, cap);
    const int* tb = bins + g * cap;
    unsigned best_d = 0xffffffffu;
    int best_f = 0x7fffffff;
    int ties = 0;
    int best_e = -1;  // bin entry (base + slot) of the winner, -1 when it came from the spill
    // Each staged chunk is sorted by (back-facing, depth lower bound) and
    // staged once: its front faces are tested first, nearest bound first, then
    // its back faces.  A triangle whose bound exceeds the pixel's current best
    // depth can neither win nor tie, and
    // neither can any triangle after it in the same run (their bounds are at
    // least as large), so a pixel stops scanning a run there.  The result is
    // the same minimum (depth, id) as one unordered pass.  Per pixel a
    // triangle is only tested when the pixel lies in its bounding box (a
    // column and a row bit mask relative to the tile) and in its conservative
    // footprint.
    //
    // Sort: 32-bit keys (facing | bound | slot) are distinct; each
    // warp sorts its 32 keys with a shuffle bitonic network, and a key's rank
    // in the chunk is its lane plus its lower bound in every other warp's
    // sorted keys (5-step binary searches).
    int n_front = 0;
    const int lane = threadIdx.x & 31;
    for (int base = 0; base < n; base += CHUNK) {
        for (int pass = 0; pass < 2; ++pass) {
            const int m = min(CHUNK, n - base);
            if (pass == 0) {
                __syncthreads();  // the previous chunk's readers are done
                bool front = false;
                unsigned key = kNoKey;
                TileTri t;
                if ((int)threadIdx.x < m) {
                    const int f = tb[base + threadIdx.x];
                    const TriView tv = tri_view[(long long)view * A.F + f];
                    front = tv.dqmin >= 0;
                    const TriFrame tf = tri_frame[(long long)b * A.F + f];
                    const int x0 = tv.x01 & 0xffff, x1 = tv.x01 >> 16;
                    const int y0 = tv.y01 & 0xffff, y1 = tv.y01 >> 16;
                    // the bound, clamped to the key's 31 - SB bits (exact below ~2^25 quanta, a
                    // lower bound above) and kept below the all-ones key of an empty slot
                    const unsigned coarse = min((unsigned)(tv.dqmin & 0x7fffffff), (1u << (31 - SB)) - 2u);
                    t.hdr = make_int4((int)bit_range(max(x0 - tx * TS, 0), min(x1 - tx * TS, TS - 1)),
                                      (int)bit_range(max(y0 - ty * TS, 0), min(y1 - ty * TS, TS - 1)),
                                      (int)coarse, f);
                    t.ea = tv.e01;
                    t.nm = make_float4(tv.num, tv.e2c.z, tv.e2c.w, tv.e2o.x);
                    t.eb = make_float4(tv.e2c.x, tv.e2c.y, 0.f, 0.f);
                    t.a = tf.a;
                    t.b = tf.b;
                    t.c = tf.c;
                    key = (front ? 0u : 0x80000000u) | (coarse << SB) | threadIdx.x;
                }
                if (threadIdx.x < CHUNK && (int)(threadIdx.x & ~31u) < m) {  // whole warps that hold keys
#pragma unroll
                    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
                        for (int stride = size >> 1; stride > 0; stride >>= 1) {
                            const unsigned o = __shfl_xor_sync(0xffffffffu, key, stride);
                            const bool keep_min = ((lane & stride) == 0) == ((lane & size) == 0);
                            key = keep_min ? min(key, o) : max(key, o);
                        }
                    }
                    s_key[threadIdx.x] = key;
                }
                n_front = __syncthreads_count(front);
                if (threadIdx.x < CHUNK && key != kNoKey) {
                    int r = lane;
                    const int me = threadIdx.x >> 5, nw = (m + 31) >> 5;
                    for (int w = 0; w < nw; ++w) {
                        if (w == me) continue;
                        const unsigned* L = s_key + 32 * w;
                        int lo = 0;
#pragma unroll
                        for (int step = 16; step > 0; step >>= 1) lo += L[lo + step] < key ? step : 0;
                        r += lo + (L[lo] < key ? 1 : 0);
                    }
                    s_rank[key & (CHUNK - 1)] = (unsigned char)r;
                }
                __syncthreads();
                if ((int)threadIdx.x < m) s_tri[s_rank[threadIdx.x]] = t;
                __syncthreads();
            }
            const int j0 = pass == 0 ? 0 : n_front;
            const int j1 = pass == 0 ? n_front : m;
            if (valid) {
                for (int slot = j0; slot < j1; ++slot) {
                    // one 16-byte header load decides whether the ray test runs
                    const int4 h = s_tri[slot].hdr;
                    if ((unsigned)h.z > best_d) break;  // neither this nor a later one can reach the best depth
                    if (!((unsigned)h.x & col_bit) || !((unsigned)h.y & row_bit)) continue;
                    const float4 ea = s_tri[slot].ea, nm = s_tri[slot].nm, eb = s_tri[slot].eb;
                    const float e0 = ea.x * cx + ea.y * cy + nm.y, e1 = ea.z * cx + ea.w * cy + nm.z,
                                e2 = eb.x * cx + eb.y * cy + nm.w;
                    if (e0 < 0.f || e1 < 0.f || e2 < 0.f) continue;  // clearly outside the projected triangle
                    int dq;
                    if (e0 >= kEdgeInterior && e1 >= kEdgeInterior && e2 >= kEdgeInterior) {
                        // clearly inside: the edge tests would pass, only the depth is needed
                        // (the same operations as ray_tri up to t)
                        const float3 n = make_float3(s_tri[slot].a.w, s_tri[slot].b.w, s_tri[slot].c.w);
                        const float ndr = dot(dir, n);
                        if (fabsf(ndr) < 0.0000001f) continue;
                        const float t = nm.x / ndr;
                        if (t < 0.f) continue;
                        dq = (int)(t * 10000.f);
                        if ((unsigned)dq > best_d) continue;
                    } else {
                        TriFrame tf;
                        tf.a = s_tri[slot].a;
                        tf.b = s_tri[slot].b;
                        tf.c = s_tri[slot].c;
                        float a, bb;
                        if (!raster_hit_below(ro_s, dir, tri_from(tf), nm.x, best_d, dq, a, bb)) continue;
                    }
                    const int f = h.w;
                    if ((unsigned)dq < best_d) {
                        best_d = (unsigned)dq;
                        best_f = f;
                        best_e = base + slot;
                        ties = 1;
                    } else {  // equal depth (deeper hits were rejected)
                        if (f < best_f) {
                            best_f = f;
                            best_e = base + slot;
                        }
                        ++ties;
                    }
                }
            }
        }
    }
    float l1s = 0.f;  // this pixel's image L1 terms (fused L1 only)
    unsigned l1c = 0;
    if (valid) {
        if (st.x > cap && st.y > 0 && st.y <= spill_tile_cap) {
            const unsigned long long key = spill_keys[(long long)(st.y - 1) * NT + threadIdx.x];
            if (key != ~0ull) {
                const unsigned kd = (unsigned)(key >> 32);
                const int kf = (int)(key & 0xffffffffu);
                if (kd < best_d) {
                    best_d = kd;
                    best_f = kf;
                    best_e = -1;
                    ties = 0;  // spilled ties are added by the diagnostics pass
                } else if (kd == best_d && kf < best_f) {
                    best_f = kf;
                    best_e = -1;
                }
            }
        }
        const long long pix = cam.pix_base + (long long)py * W + px;
        if (best_d == 0xffffffffu) {
            A.face[pix] = -1;
            A.bary[2 * pix + 0] = 0.f;
            A.bary[2 * pix + 1] = 0.f;
            A.render[3 * pix + 0] = 0.f;
            A.render[3 * pix + 1] = 0.f;
            A.render[3 * pix + 2] = 0.f;
            if (A.depth_q) A.depth_q[pix] = 0x7fffffff;
            if (TIES) A.tie_count[pix] = 0;
        } else {
            // the fused L1's target, loaded before this pixel's stores (which
            // the compiler may not move it past)
            const bool l1m = A.l1_sum && (!A.l1_mask || A.l1_mask[pix]);
            const float3 tg = l1m ? ld3(A.l1_target + 3 * pix) : make_float3(0.f, 0.f, 0.f);
            // recompute the winner's barycentrics (same arithmetic as the hit test)
            // the winner's triangle and plane offset: from the staged chunk when
            // the winner is in the last one staged (s_tri is rewritten only
            // after the next tile's first barrier), else from global memory
            const int last_base = n > 0 ? ((n - 1) / CHUNK) * CHUNK : 0;
            TriS Tw;
            float wnum;
            if (best_e >= last_base) {
                const TileTri& w = s_tri[best_e - last_base];
                TriFrame tf;
                tf.a = w.a;
                tf.b = w.b;
                tf.c = w.c;
                Tw = tri_from(tf);
                wnum = w.nm.x;
            } else {
                Tw = tri_from(tri_frame[(long long)b * A.F + best_f]);
                wnum = tri_view[(long long)view * A.F + best_f].num;
            }
            float a, bb;
            winner_bary(ro_s, dir, Tw, wnum, a, bb);
            // every load of the shading before the first store of the pixel
            const float3 col = shade_pixel(A, cam, view, b, best_f, a, bb, dir);
            A.face[pix] = best_f;
            A.bary[2 * pix + 0] = a;
            A.bary[2 * pix + 1] = bb;
            A.render[3 * pix + 0] = col.x;
            A.render[3 * pix + 1] = col.y;
            A.render[3 * pix + 2] = col.z;
            if (A.depth_q) A.depth_q[pix] = (int)best_d;
            if (TIES) A.tie_count[pix] = ties;
            if (l1m) {
                const float d0 = l1_diff(col.x, tg.x), d1 = l1_diff(col.y, tg.y), d2 = l1_diff(col.z, tg.z);
                l1s = fabsf(d0) + fabsf(d1) + fabsf(d2);
                l1c = (d0 != 0.f) + (d1 != 0.f) + (d2 != 0.f);
            }
        }
    }
    if (A.l1_sum) {  // launch-uniform: each warp's partial L1 sum and count
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            l1s += __shfl_xor_sync(0xffffffffu, l1s, o);
            l1c += __shfl_xor_sync(0xffffffffu, l1c, o);
        }
        if (lane == 0) {
            A.l1_sum[g * (NT / 32) + (threadIdx.x >> 5)] = l1s;
            A.l1_cnt[g * (NT / 32) + (threadIdx.x >> 5)] = l1c;
        }
    }
    }
}

// the fused L1's warp partials summed into the L1 state (zeroed before)
__global__ void k_l1_tiles(long long n, const float* __restrict__ sums, const unsigned* __restrict__ cnts,
                           L1State* __restrict__ state) {
    double s = 0.0;
    unsigned long long c = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        s += sums[i];
        c += cnts[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0 && (s != 0.0 || c != 0)) {
        atomicAdd(&state->sum, s);
        atomicAdd(&state->count, c);
    }
}

__global__ void k_l1_loss(const L1State* __restrict__ state, float* __restrict__ loss) {
    const unsigned long long c = state->count;
    *loss = c ? (float)(state->sum / (double)c) : 0.f;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// grid of a persistent kernel: as many CTAs as are resident at once (SMs x
// CTAs per SM), never more than the work items
template <typename K>
static unsigned resident_grid(K kernel, int threads, long long items) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    return (unsigned)std::max<long long>(1, std::min((long long)sms * per_sm, items));
}
// Per-camera layout of a frame for the current tile size: each camera's
// resolution, tile grids and offsets, and the camera of every tile (the tile
// resolve and the adjoint launch one CTA per tile of the whole call).
hc_status raster_layout(RasterWorkspace& ws) {
    const int TS = ws.tile, C = (int)ws.cam_w.size();
    if (ws.layout_tile == TS) return HC_OK;
    std::vector<CamLayout> L(C);
    std::vector<int> tc, tcb;
    long long pix = 0, tile = 0, tile_b = 0;
    for (int c = 0; c < C; ++c) {
        CamLayout& l = L[c];
        l.W = ws.cam_w[c];
        l.H = ws.cam_h[c];
        l.tiles_x = div_up(l.W, TS);
        l.tiles_x_b = div_up(l.W, kAdjointTile);
        l.fd_tiles_x = FastDiv((unsigned)l.tiles_x);
        l.fd_tiles_x_b = FastDiv((unsigned)l.tiles_x_b);
        l.pix = pix;
        l.tile = tile;
        l.tile_b = tile_b;
        const long long nt = (long long)l.tiles_x * div_up(l.H, TS);
        const long long ntb = (long long)l.tiles_x_b * div_up(l.H, kAdjointTile);
        tc.insert(tc.end(), (size_t)nt, c);
        tcb.insert(tcb.end(), (size_t)ntb, c);
        pix += (long long)l.W * l.H;
        tile += nt;
        tile_b += ntb;
    }
    HC_TRY(upload(ws.layout, L.data(), L.size()));
    HC_TRY(upload(ws.tile_cam, tc.data(), tc.size()));
    HC_TRY(upload(ws.tile_cam_b, tcb.data(), tcb.size()));
    ws.P_frame = pix;
    ws.T_frame = tile;
    ws.Tb_frame = tile_b;
    ws.layout_tile = TS;
    ws.cap_views = 0;  // bins depend on the tile count
    return HC_OK;
}

hc_status raster_reserve(RasterWorkspace& ws, int views, int F) {
    HC_TRY(raster_layout(ws));
    const int TS = ws.tile;
    const int C = (int)ws.cam_w.size();
    const long long tiles = (long long)(views / C) * ws.T_frame;  // all tiles of the call
    if (views > ws.cap_views || ws.bins.bytes < (size_t)tiles * ws.bin_cap * sizeof(int)) {
        HC_TRY(ws.cams.ensure(sizeof(ViewCam) * views));
        HC_TRY(ws.tri_view.ensure(sizeof(TriView) * (size_t)views * F));
        HC_TRY(ws.tile_state.ensure(sizeof(int2) * (size_t)tiles));
        HC_TRY(ws.bins.ensure(sizeof(int) * (size_t)tiles * ws.bin_cap));
        // crumpled meshes overflow many bins: room for four spilled pairs per
        // (view, triangle), and a key block for every tile while that stays
        // under 4 GB (a quarter of the tiles beyond); overflow is reported by
        // hc_renderer_stats
        ws.spill_cap = std::max<long long>(1 << 22, 4ll * views * F);
        HC_TRY(ws.spill.ensure(sizeof(int2) * (size_t)ws.spill_cap));
        const long long per_tile = (long long)TS * TS * sizeof(unsigned long long);
        ws.spill_tile_cap = (int)(tiles * per_tile <= (4ll << 30) ? tiles : std::max<long long>(256, tiles / 4));
        HC_TRY(ws.spill_keys.ensure(sizeof(unsigned long long) * (size_t)ws.spill_tile_cap * TS * TS));
        HC_TRY(ws.stats.ensure(sizeof(RasterStats)));
        ws.cap_views = views;
    }
    return HC_OK;
}

hc_status raster_forward(const Topology& topo, RasterWorkspace& ws, cudaStream_t s, int B, int C, int albedo,
                         int shading, const float* verts, const float* colors, const float* texture, int tex_h,
                         int tex_w, const float* sh, const float* extr, const float* intr, float* bary, int* face,
                         float* render, float* vnormal, int* depth_q, int* tie_count, const L1Fuse* l1) {
    const int V = B * C;
    const int N = topo.N, F = topo.F;
    HC_TRY(raster_reserve(ws, V, F));
    HC_TRY(ws.tri_frame.ensure(sizeof(TriFrame) * (size_t)B * F));
    HC_TRY(ws.proj.ensure(sizeof(float4) * (size_t)V * N));
    const int TS = ws.tile;
    const long long tiles = (long long)B * ws.T_frame;
    ViewCam* cams = ws.cams.as<ViewCam>();
    TriFrame* tf = ws.tri_frame.as<TriFrame>();
    TriView* tv = ws.tri_view.as<TriView>();
    int2* tstate = ws.tile_state.as<int2>();
    RasterStats* stats = ws.stats.as<RasterStats>();

    HC_CUDA(cudaMemsetAsync(tstate, 0, sizeof(int2) * (size_t)tiles, s));
    HC_CUDA(cudaMemsetAsync(stats, 0, sizeof(RasterStats), s));
    ws.clock.begin(kKViewSetup, s);
    k_view_setup<<<div_up(V, 64), 64, 0, s>>>(V, C, extr, intr, ws.layout.as<CamLayout>(), ws.P_frame, ws.T_frame,
                                              ws.Tb_frame, cams);
    HC_CHECK_LAUNCH();
    ws.clock.end(kKViewSetup, s);
    ws.clock.begin(kKVertexNormals, s);
    k_vertex_normals<<<div_up((long long)B * N, 256), 256, 0, s>>>(
        B, C, N, topo.faces.as<int3>(), topo.vf.as<int>(), topo.vf_id.as<int2>(), verts, vnormal);
    HC_CHECK_LAUNCH();
    ws.clock.end(kKVertexNormals, s);
    ws.clock.begin(kKTriFrame, s);
    k_tri_frame<<<div_up((long long)B * F, 256), 256, 0, s>>>(B, F, N, topo.faces.as<int3>(), verts, tf);
    HC_CHECK_LAUNCH();
    ws.clock.end(kKTriFrame, s);
    ws.clock.begin(kKBin, s);
    k_project_vertices<<<div_up((long long)V * N, 256), 256, 0, s>>>(V, C, N, verts, cams, ws.proj.as<float4>());
    HC_CHECK_LAUNCH();
    HC_REQUIRE(V <= 65535, "too many views in one call (%d)", V);
    HC_REQUIRE(tiles < (1ll << 31), "too many tiles in one call (%lld)", tiles);
    const int ts_shift = TS == 8 ? 3 : (TS == 16 ? 4 : 5);
    HC_REQUIRE(TS == (1 << ts_shift), "tile size %d is not 8, 16 or 32", TS);
    k_bin<<<dim3(div_up(F, 256), V), 256, 0, s>>>(
        V, C, F, N, TS, ts_shift, ws.bin_cap, topo.faces.as<int3>(), ws.proj.as<float4>(), cams, tf, tv, tstate,
        ws.bins.as<int>(),
        ws.spill.as<int2>(), ws.spill_cap, ws.spill_keys.as<unsigned long long>(), ws.spill_tile_cap, stats);
    HC_CHECK_LAUNCH();
    ws.clock.end(kKBin, s);
    ws.clock.begin(kKSpill, s);
    k_spill<<<148 * 4, 128, 0, s>>>(C, F, TS, ws.T_frame, ws.tile_cam.as<int>(), cams, tf, tv, tstate,
                                    ws.spill.as<int2>(), ws.spill_cap,
                                    ws.spill_tile_cap, ws.spill_keys.as<unsigned long long>(), stats, nullptr,
                                    nullptr);
    HC_CHECK_LAUNCH();
    ws.clock.end(kKSpill, s);
    ShadeArgs A;
    A.B = B;
    A.C = C;
    A.N = N;
    A.F = F;
    A.proj = ws.proj.as<float4>();
    A.albedo = albedo;
    A.shading = shading;
    A.faces = topo.faces.as<int3>();
    A.texcoords = topo.texcoords.as<float>();
    A.verts = verts;
    A.colors = colors;
    A.texture = texture;
    A.tex_w = tex_w;
    A.tex_h = tex_h;
    A.sh = sh;
    A.vnormal = vnormal;
    A.bary = bary;
    A.face = face;
    A.render = render;
    A.depth_q = depth_q;
    A.tie_count = tie_count;
    A.l1_target = nullptr;
    A.l1_mask = nullptr;
    A.l1_sum = nullptr;
    A.l1_cnt = nullptr;
    const long long l1_n = tiles * (TS * TS / 32);  // warp partials of the fused L1
    if (l1) {
        HC_TRY(ws.l1_part.ensure(8 * (size_t)l1_n));
        HC_CUDA(cudaMemsetAsync(l1->state, 0, sizeof(L1State), s));
        A.l1_target = l1->target;
        A.l1_mask = l1->mask;
        A.l1_sum = ws.l1_part.as<float>();
        A.l1_cnt = reinterpret_cast<unsigned*>(A.l1_sum + l1_n);
    }
    const int* tcam = ws.tile_cam.as<int>();
    HC_REQUIRE(tiles < (1ll << 31), "too many tiles in one call (%lld)", tiles);
    HC_TRY(ws.claim.ensure(sizeof(unsigned long long)));
    unsigned long long* claim = ws.claim.as<unsigned long long>();
    HC_CUDA(cudaMemsetAsync(claim, 0, sizeof(unsigned long long), s));
    const int* kbins = ws.bins.as<int>();
    const unsigned long long* kspill = ws.spill_keys.as<unsigned long long>();
    ws.clock.begin(kKResolve, s);
#define HC_RESOLVE_CASE(TSV)                                                                                   \
    case TSV:                                                                                                  \
        if (A.tie_count)                                                                                       \
            k_resolve<TSV, true><<<resident_grid(k_resolve<TSV, true>, TSV * TSV, tiles), TSV * TSV, 0, s>>>(  \
                A, FastDiv((unsigned)ws.T_frame), tcam, ws.bin_cap, cams, tf, tv, tstate, kbins, kspill,       \
                ws.spill_tile_cap, tiles, claim);                                                              \
        else                                                                                                   \
            k_resolve<TSV, false><<<resident_grid(k_resolve<TSV, false>, TSV * TSV, tiles), TSV * TSV, 0, s>>>( \
                A, FastDiv((unsigned)ws.T_frame), tcam, ws.bin_cap, cams, tf, tv, tstate, kbins, kspill,       \
                ws.spill_tile_cap, tiles, claim);                                                              \
        break;
    switch (TS) {
        HC_RESOLVE_CASE(8)
        HC_RESOLVE_CASE(16)
        HC_RESOLVE_CASE(32)
        default:
            HC_FAIL(HC_ERR_INVALID, "unsupported tile size %d", TS);
    }
#undef HC_RESOLVE_CASE
    HC_CHECK_LAUNCH();
    ws.clock.end(kKResolve, s);
    if (l1) {
        k_l1_tiles<<<148 * 2, 256, 0, s>>>(l1_n, A.l1_sum, A.l1_cnt, l1->state);
        HC_CHECK_LAUNCH();
        if (l1->loss) {
            k_l1_loss<<<1, 1, 0, s>>>(l1->state, l1->loss);
            HC_CHECK_LAUNCH();
        }
    }
    if (tie_count && depth_q) {
        k_spill<<<148 * 4, 128, 0, s>>>(C, F, TS, ws.T_frame, ws.tile_cam.as<int>(), cams, tf, tv, tstate,
                                    ws.spill.as<int2>(), ws.spill_cap,
                                        ws.spill_tile_cap, ws.spill_keys.as<unsigned long long>(), stats, depth_q,
                                        tie_count);
        HC_CHECK_LAUNCH();
    }
    return HC_OK;
}

}  // namespace hc
