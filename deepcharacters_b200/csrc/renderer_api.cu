// C-ABI entry points of the renderer (hc_renderer_*).
#include <string.h>

#include <algorithm>
#include <vector>

#include "renderer.cuh"

namespace hc {

hc_status raster_forward(const Topology& topo, RasterWorkspace& ws, cudaStream_t s, int B, int C, int albedo,
                         int shading, const float* verts, const float* colors, const float* texture, int tex_h,
                         int tex_w, const float* sh, const float* extr, const float* intr, float* bary, int* face,
                         float* render, float* vnormal, int* depth_q, int* tie_count,
                         const L1Fuse* l1 = nullptr);
hc_status raster_reserve(RasterWorkspace& ws, int views, int F);
hc_status raster_uv_maps(const Topology& topo, UvTable& tab, cudaStream_t s, int B, int C, long long P_frame, int mode,
                         const float* verts, int tex_h, int tex_w, float* bary, int* face, float* render,
                         float* vnormal, float* uv_map);
hc_status raster_backward(const Topology& topo, RasterWorkspace& ws, DevBuf& nrm_ws, cudaStream_t s, int B, int C,
                          int albedo, int shading, int ifs, int tfs, const float* grad, const float* verts,
                          const float* colors, const float* texture, int tex_h, int tex_w, const float* sh,
                          const float* target, const float* vnormal, const float* bary, const int* face,
                          const float* extr, const float* intr, float* vpos_grad, float* vcol_grad, float* tex_grad,
                          float* sh_grad, int parity, const L1Fuse* l1 = nullptr);

static int parse_albedo(const char* m) {
    if (!m) return -1;
    static const char* names[] = {"vertexColor", "textured", "normal", "lighting", "foregroundMask",
                                  "position", "depth", "uv", "texturedBilinear"};
    for (int i = 0; i < 9; ++i)
        if (!strcmp(m, names[i])) return i;
    return -1;
}

static int parse_shading(const char* m) {
    if (!m) return -1;
    if (!strcmp(m, "shaded")) return kShaded;
    if (!strcmp(m, "shadeless")) return kShadeless;
    return -1;
}

static int parse_normal_map(const char* m) {
    if (!m || !strcmp(m, "none")) return kNmNone;
    if (!strcmp(m, "normal")) return kNmOriginal;
    if (!strcmp(m, "position")) return kNmHitPosition;
    if (!strcmp(m, "face")) return kNmFace;
    return -1;
}

// Vertex -> incident faces in increasing face order, by counting sort
// (the reference builds the same lists with an O(N*F) scan,
// CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cpp:154-183).  A face
// that names a vertex twice is listed once for it.  Vertices without faces get
// an empty range (the reference drops them from the offset table).
void build_vertex_faces(int N, const int32_t* faces, int F, std::vector<int>& vf, std::vector<int>& vf_id) {
    std::vector<int> cnt(N + 1, 0);
    for (int f = 0; f < F; ++f) {
        const int a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
        cnt[a]++;
        if (b != a) cnt[b]++;
        if (c != a && c != b) cnt[c]++;
    }
    vf_id.assign(2 * (size_t)N, 0);
    std::vector<int> start(N + 1, 0);
    for (int v = 0; v < N; ++v) start[v + 1] = start[v] + cnt[v];
    for (int v = 0; v < N; ++v) {
        vf_id[2 * v] = start[v];
        vf_id[2 * v + 1] = cnt[v];
    }
    vf.assign(start[N], 0);
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int f = 0; f < F; ++f) {
        const int a = faces[3 * f], b = faces[3 * f + 1], c = faces[3 * f + 2];
        vf[fill[a]++] = f;
        if (b != a) vf[fill[b]++] = f;
        if (c != a && c != b) vf[fill[c]++] = f;
    }
}

hc_status topology_upload(Topology& t, int N, const int32_t* faces, int F, const float* texcoords, int n_tc) {
    for (int i = 0; i < 3 * F; ++i)
        HC_REQUIRE(faces[i] >= 0 && faces[i] < N, "face %d references vertex %d outside [0,%d)", i / 3, faces[i], N);
    std::vector<int> vf, vf_id;
    build_vertex_faces(N, faces, F, vf, vf_id);
    t.N = N;
    t.F = F;
    HC_TRY(upload(t.faces, faces, (size_t)3 * F));
    HC_TRY(upload(t.vf, vf.data(), vf.size()));
    HC_TRY(upload(t.vf_id, vf_id.data(), vf_id.size()));
    if (texcoords && n_tc == 6 * F) {
        HC_TRY(upload(t.texcoords, texcoords, (size_t)6 * F));
        t.has_texcoords = true;
    } else {
        // modes that sample UVs read zeros
        std::vector<float> z((size_t)6 * F, 0.f);
        HC_TRY(upload(t.texcoords, z.data(), z.size()));
        t.has_texcoords = false;
    }
    return HC_OK;
}

}  // namespace hc

struct hc_renderer_s {
    hc::Topology topo;
    hc::RasterWorkspace ws;
    hc::DevBuf nrm_grad;  // backward: gradient w.r.t. unnormalised vertex normals
    hc::UvTable uv;       // texel table of the UV-space maps
    int C = 0, W = 0, H = 0;
    int albedo = 0, shading = 0, normal_map = hc::kNmNone;
    int image_filter = 2, texture_filter = 2;
    int grad_parity = 0;  // 1: the reference's barycentric-Jacobian formula
};

using namespace hc;

static long long frame_pixels(const hc_renderer_s* h) {
    long long p = 0;
    for (size_t c = 0; c < h->ws.cam_w.size(); ++c) p += (long long)h->ws.cam_w[c] * h->ws.cam_h[c];
    return p;
}

extern "C" hc_status hc_renderer_create(hc_renderer* out, const int32_t* faces, int32_t n_faces,
                                        const float* texture_coordinates, int32_t n_texcoords,
                                        int32_t number_of_vertices, int32_t number_of_cameras,
                                        int32_t render_resolution_u, int32_t render_resolution_v,
                                        const char* albedo_mode, const char* shading_mode,
                                        int32_t image_filter_size, int32_t texture_filter_size,
                                        const char* compute_normal_map) {
    clear_error();
    HC_REQUIRE(out, "out is NULL");
    *out = nullptr;
    HC_REQUIRE(faces && n_faces > 0, "faces must be non-empty");
    HC_REQUIRE(number_of_vertices > 0, "number_of_vertices not set (%d)", number_of_vertices);
    HC_REQUIRE(number_of_cameras > 0, "number_of_cameras not set (%d)", number_of_cameras);
    HC_REQUIRE(render_resolution_u > 0 && render_resolution_u < 32768, "render_resolution_u out of range (%d)",
               render_resolution_u);
    HC_REQUIRE(render_resolution_v > 0 && render_resolution_v < 32768, "render_resolution_v out of range (%d)",
               render_resolution_v);
    const int albedo = parse_albedo(albedo_mode);
    HC_REQUIRE(albedo >= 0, "INVALID ALBEDO MODE '%s'", albedo_mode ? albedo_mode : "(null)");
    int shading = parse_shading(shading_mode);
    HC_REQUIRE(shading >= 0, "INVALID SHADING MODE '%s'", shading_mode ? shading_mode : "(null)");
    const int nm = parse_normal_map(compute_normal_map);
    HC_REQUIRE(nm >= 0, "INVALID Normal MODE '%s'", compute_normal_map);
    HC_REQUIRE(n_texcoords == 0 || n_texcoords == 6 * n_faces,
               "texture_coordinates has %d values, expected 6 per face (%d)", n_texcoords, 6 * n_faces);
    // the reference op forces shadeless for every mode but vertexColor / textured
    // (CudaRenderer/cpp/src/TensorflowOperators/CudaRenderer/CudaRenderer.cpp:70-74)
    if (albedo != kVertexColor && albedo != kTextured && albedo != kTexturedBilinear) shading = kShadeless;
    hc_renderer_s* r = new hc_renderer_s();
    hc_status st = topology_upload(r->topo, number_of_vertices, faces, n_faces, texture_coordinates, n_texcoords);
    if (st != HC_OK) {
        delete r;
        return st;
    }
    r->C = number_of_cameras;
    r->W = render_resolution_u;
    r->H = render_resolution_v;
    r->ws.cam_w.assign(number_of_cameras, render_resolution_u);
    r->ws.cam_h.assign(number_of_cameras, render_resolution_v);
    r->albedo = albedo;
    r->shading = shading;
    r->normal_map = nm;
    r->image_filter = image_filter_size;
    r->texture_filter = texture_filter_size;
    *out = r;
    return HC_OK;
}

static void release_all(hc_renderer_s* r) {
    if (r->ws.clock.made)
        for (cudaEvent_t& e : r->ws.clock.ev) cudaEventDestroy(e);
    r->ws.clock.made = false;
    DevBuf* bufs[] = {&r->topo.faces, &r->topo.vf, &r->topo.vf_id, &r->topo.texcoords,
                      &r->ws.cams, &r->ws.tri_frame, &r->ws.tri_view, &r->ws.tile_state,
                      &r->ws.bins, &r->ws.spill, &r->ws.spill_keys, &r->ws.stats, &r->nrm_grad,
                      &r->uv.faces, &r->uv.table, &r->ws.layout, &r->ws.tile_cam, &r->ws.tile_cam_b, &r->ws.proj,
                      &r->ws.l1_part, &r->ws.claim};
    for (DevBuf* b : bufs) b->release();
}

extern "C" hc_status hc_renderer_destroy(hc_renderer h) {
    clear_error();
    if (!h) return HC_OK;
    release_all(h);
    delete h;
    return HC_OK;
}

extern "C" hc_status hc_renderer_reserve(hc_renderer h, int32_t batch) {
    clear_error();
    HC_REQUIRE(h && batch > 0, "invalid handle or batch");
    HC_TRY(raster_reserve(h->ws, batch * h->C, h->topo.F));
    HC_TRY(h->ws.tri_frame.ensure(sizeof(TriFrame) * (size_t)batch * h->topo.F));
    HC_TRY(h->ws.proj.ensure(sizeof(float4) * (size_t)batch * h->C * h->topo.N));
    return HC_OK;
}

extern "C" hc_status hc_renderer_set_tuning(hc_renderer h, int32_t tile, int32_t bin_capacity) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(tile == 8 || tile == 16 || tile == 32, "tile must be 8, 16 or 32 (got %d)", tile);
    HC_REQUIRE(bin_capacity >= 1 && bin_capacity <= (1 << 16), "bin_capacity out of range (%d)", bin_capacity);
    if (tile != h->ws.tile || bin_capacity != h->ws.bin_cap) {
        h->ws.tile = tile;
        h->ws.bin_cap = bin_capacity;
        h->ws.cap_views = 0;  // re-derive tile grid and bin sizes on the next reserve
        h->ws.bins.release();
        h->ws.tile_state.release();
        h->ws.spill_keys.release();
    }
    return HC_OK;
}

extern "C" hc_status hc_renderer_forward_ex(hc_renderer h, void* stream, int32_t batch, const float* vertex_pos,
                                            const float* vertex_color, const float* texture,
                                            int32_t texture_height, int32_t texture_width, const float* sh_coeff,
                                            const float* extrinsics, const float* intrinsics,
                                            float* barycentric_buffer, int32_t* face_buffer, float* render_buffer,
                                            float* vertex_normal, float* normal_map, int32_t* depth_q,
                                            int32_t* tie_count) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(batch > 0, "batch must be positive (%d)", batch);
    HC_REQUIRE(vertex_pos && extrinsics && intrinsics && barycentric_buffer && face_buffer && render_buffer &&
                   vertex_normal,
               "NULL input/output pointer");
    if (h->albedo == kVertexColor) HC_REQUIRE(vertex_color, "vertexColor mode needs vertex_color");
    if (h->albedo == kTextured || h->albedo == kTexturedBilinear) {
        HC_REQUIRE(texture && texture_width > 0 && texture_height > 0, "textured mode needs a texture");
        HC_REQUIRE(h->topo.has_texcoords, "textured mode needs texture_coordinates");
    }
    const bool needs_sh = (h->shading == kShaded && h->albedo != kNormal) || h->albedo == kLighting;
    if (needs_sh) HC_REQUIRE(sh_coeff, "shading needs sh_coeff");
    cudaStream_t s = (cudaStream_t)stream;
    if (h->normal_map != kNmNone)
        return raster_uv_maps(h->topo, h->uv, s, batch, h->C, frame_pixels(h), h->normal_map, vertex_pos, texture_height,
                              texture_width, barycentric_buffer, face_buffer, render_buffer, vertex_normal,
                              normal_map);
    return raster_forward(h->topo, h->ws, s, batch, h->C, h->albedo, h->shading, vertex_pos,
                          vertex_color, texture, texture_height, texture_width, sh_coeff, extrinsics, intrinsics,
                          barycentric_buffer, face_buffer, render_buffer, vertex_normal, depth_q, tie_count);
}

extern "C" hc_status hc_renderer_forward(hc_renderer h, void* stream, int32_t batch, const float* vertex_pos,
                                         const float* vertex_color, const float* texture, int32_t texture_height,
                                         int32_t texture_width, const float* sh_coeff, const float* extrinsics,
                                         const float* intrinsics, float* barycentric_buffer, int32_t* face_buffer,
                                         float* render_buffer, float* vertex_normal, float* normal_map) {
    return hc_renderer_forward_ex(h, stream, batch, vertex_pos, vertex_color, texture, texture_height,
                                  texture_width, sh_coeff, extrinsics, intrinsics, barycentric_buffer, face_buffer,
                                  render_buffer, vertex_normal, normal_map, nullptr, nullptr);
}

extern "C" hc_status hc_renderer_stats(hc_renderer h, void* stream, int64_t* binned, int64_t* spilled) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    RasterStats st;
    memset(&st, 0, sizeof(st));
    if (h->ws.stats.ptr) {
        HC_CUDA(cudaMemcpyAsync(&st, h->ws.stats.ptr, sizeof(st), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
        HC_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    }
    if (binned) *binned = (int64_t)st.binned;
    if (spilled) *spilled = (int64_t)st.spilled;
    if (st.overflow & 4) HC_FAIL(HC_ERR_CUDA, "a target copy of the raster adjoint did not complete (flags %d)",
                                 st.overflow);
    if (st.overflow) HC_FAIL(HC_ERR_OVERFLOW, "raster spill capacity exceeded (flags %d)", st.overflow);
    return HC_OK;
}

extern "C" hc_status hc_renderer_backward(hc_renderer h, void* stream, int32_t batch, const float* render_buffer_grad,
                                          const float* vertex_pos, const float* vertex_color, const float* texture,
                                          int32_t texture_height, int32_t texture_width, const float* sh_coeff,
                                          const float* target_image, const float* vertex_normal,
                                          const float* barycentric_buffer, const int32_t* face_buffer,
                                          const float* extrinsics, const float* intrinsics, float* vertex_pos_grad,
                                          float* vertex_color_grad, float* texture_grad, float* sh_coeff_grad) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(batch > 0, "batch must be positive (%d)", batch);
    HC_REQUIRE(h->albedo == kVertexColor || h->albedo == kTextured || h->albedo == kTexturedBilinear,
               "renderer gradients exist only for vertexColor and textured albedo");
    HC_REQUIRE(render_buffer_grad && vertex_pos && target_image && vertex_normal && barycentric_buffer &&
                   face_buffer && extrinsics && intrinsics && vertex_pos_grad,
               "NULL input/output pointer");
    if (h->albedo == kVertexColor) HC_REQUIRE(vertex_color && vertex_color_grad, "vertexColor mode needs colours");
    if (h->albedo == kTextured || h->albedo == kTexturedBilinear)
        HC_REQUIRE(texture && texture_grad && texture_width > 0 && texture_height > 0, "textured mode needs a texture");
    if (h->shading == kShaded) HC_REQUIRE(sh_coeff && sh_coeff_grad, "shaded mode needs sh_coeff");
    return raster_backward(h->topo, h->ws, h->nrm_grad, (cudaStream_t)stream, batch, h->C, h->albedo,
                           h->shading, h->image_filter, h->texture_filter, render_buffer_grad, vertex_pos,
                           vertex_color, texture, texture_height, texture_width, sh_coeff, target_image,
                           vertex_normal, barycentric_buffer, face_buffer, extrinsics, intrinsics, vertex_pos_grad,
                           vertex_color_grad, texture_grad, sh_coeff_grad, h->grad_parity);
}

extern "C" hc_status hc_renderer_forward_l1(hc_renderer h, void* stream, int32_t batch, const float* vertex_pos,
                                            const float* vertex_color, const float* texture,
                                            int32_t texture_height, int32_t texture_width, const float* sh_coeff,
                                            const float* extrinsics, const float* intrinsics,
                                            float* barycentric_buffer, int32_t* face_buffer, float* render_buffer,
                                            float* vertex_normal, const float* target_image,
                                            const uint8_t* foreground_mask, void* l1_state, float* loss) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(batch > 0, "batch must be positive (%d)", batch);
    HC_REQUIRE(h->normal_map == kNmNone, "the fused L1 needs compute_normal_map = none");
    HC_REQUIRE(vertex_pos && extrinsics && intrinsics && barycentric_buffer && face_buffer && render_buffer &&
                   vertex_normal && target_image && l1_state,
               "NULL input/output pointer");
    if (h->albedo == kVertexColor) HC_REQUIRE(vertex_color, "vertexColor mode needs vertex_color");
    if (h->albedo == kTextured || h->albedo == kTexturedBilinear) {
        HC_REQUIRE(texture && texture_width > 0 && texture_height > 0, "textured mode needs a texture");
        HC_REQUIRE(h->topo.has_texcoords, "textured mode needs texture_coordinates");
    }
    const bool needs_sh = (h->shading == kShaded && h->albedo != kNormal) || h->albedo == kLighting;
    if (needs_sh) HC_REQUIRE(sh_coeff, "shading needs sh_coeff");
    L1Fuse l1;
    l1.target = target_image;
    l1.mask = foreground_mask;
    l1.state = static_cast<L1State*>(l1_state);
    l1.loss = loss;
    return raster_forward(h->topo, h->ws, (cudaStream_t)stream, batch, h->C, h->albedo, h->shading, vertex_pos,
                          vertex_color, texture, texture_height, texture_width, sh_coeff, extrinsics, intrinsics,
                          barycentric_buffer, face_buffer, render_buffer, vertex_normal, nullptr, nullptr, &l1);
}

extern "C" hc_status hc_renderer_backward_l1(hc_renderer h, void* stream, int32_t batch, const void* l1_state,
                                             const float* render_buffer, const uint8_t* foreground_mask,
                                             const float* vertex_pos, const float* vertex_color,
                                             const float* texture, int32_t texture_height, int32_t texture_width,
                                             const float* sh_coeff, const float* target_image,
                                             const float* vertex_normal, const float* barycentric_buffer,
                                             const int32_t* face_buffer, const float* extrinsics,
                                             const float* intrinsics, float* vertex_pos_grad,
                                             float* vertex_color_grad, float* texture_grad, float* sh_coeff_grad) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    HC_REQUIRE(batch > 0, "batch must be positive (%d)", batch);
    HC_REQUIRE(h->albedo == kVertexColor || h->albedo == kTextured || h->albedo == kTexturedBilinear,
               "renderer gradients exist only for vertexColor and textured albedo");
    HC_REQUIRE(l1_state && render_buffer && vertex_pos && target_image && vertex_normal && barycentric_buffer &&
                   face_buffer && extrinsics && intrinsics && vertex_pos_grad,
               "NULL input/output pointer");
    if (h->albedo == kVertexColor) HC_REQUIRE(vertex_color && vertex_color_grad, "vertexColor mode needs colours");
    if (h->albedo == kTextured || h->albedo == kTexturedBilinear)
        HC_REQUIRE(texture && texture_grad && texture_width > 0 && texture_height > 0, "textured mode needs a texture");
    if (h->shading == kShaded) HC_REQUIRE(sh_coeff && sh_coeff_grad, "shaded mode needs sh_coeff");
    L1Fuse l1;
    l1.target = target_image;
    l1.mask = foreground_mask;
    l1.state = const_cast<L1State*>(static_cast<const L1State*>(l1_state));
    l1.render = render_buffer;
    return raster_backward(h->topo, h->ws, h->nrm_grad, (cudaStream_t)stream, batch, h->C, h->albedo,
                           h->shading, h->image_filter, h->texture_filter, nullptr, vertex_pos, vertex_color, texture,
                           texture_height, texture_width, sh_coeff, target_image, vertex_normal, barycentric_buffer,
                           face_buffer, extrinsics, intrinsics, vertex_pos_grad, vertex_color_grad, texture_grad,
                           sh_coeff_grad, h->grad_parity, &l1);
}

extern "C" hc_status hc_renderer_set_gradient_parity(hc_renderer h, int32_t parity) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    h->grad_parity = parity ? 1 : 0;
    return HC_OK;
}

extern "C" hc_status hc_renderer_set_adjoint_schedule(hc_renderer h, int32_t dynamic) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    h->ws.adjoint_dynamic = dynamic ? 1 : 0;
    return HC_OK;
}

extern "C" hc_status hc_renderer_set_kernel_timing(hc_renderer h, int32_t enable) {
    clear_error();
    HC_REQUIRE(h, "invalid handle");
    KernelClock& c = h->ws.clock;
    if (enable && !c.made) {
        for (cudaEvent_t& e : c.ev) HC_CUDA(cudaEventCreate(&e));
        c.made = true;
    }
    c.on = enable != 0;
    c.recorded = 0;
    return HC_OK;
}

extern "C" hc_status hc_renderer_kernel_times(hc_renderer h, float* ms, int32_t n) {
    clear_error();
    HC_REQUIRE(h && ms && n >= 0, "invalid arguments");
    KernelClock& c = h->ws.clock;
    for (int k = 0; k < n; ++k) {
        ms[k] = -1.f;
        if (k < kKCount && c.made && (c.recorded >> k & 1u)) {
            HC_CUDA(cudaEventSynchronize(c.ev[2 * k + 1]));
            HC_CUDA(cudaEventElapsedTime(&ms[k], c.ev[2 * k], c.ev[2 * k + 1]));
        }
    }
    c.recorded = 0;
    return HC_OK;
}

extern "C" hc_status hc_renderer_create_multires(hc_renderer* out, const int32_t* faces, int32_t n_faces,
                                                 const float* texture_coordinates, int32_t n_texcoords,
                                                 int32_t number_of_vertices, int32_t number_of_cameras,
                                                 const int32_t* camera_widths, const int32_t* camera_heights,
                                                 const char* albedo_mode, const char* shading_mode,
                                                 int32_t image_filter_size, int32_t texture_filter_size,
                                                 const char* compute_normal_map) {
    clear_error();
    HC_REQUIRE(out, "out is NULL");
    *out = nullptr;
    HC_REQUIRE(camera_widths && camera_heights && number_of_cameras > 0, "camera sizes must be given");
    for (int c = 0; c < number_of_cameras; ++c)
        HC_REQUIRE(camera_widths[c] > 0 && camera_widths[c] < 32768 && camera_heights[c] > 0 &&
                       camera_heights[c] < 32768,
                   "camera %d size %dx%d out of range", c, camera_widths[c], camera_heights[c]);
    HC_TRY(hc_renderer_create(out, faces, n_faces, texture_coordinates, n_texcoords, number_of_vertices,
                              number_of_cameras, camera_widths[0], camera_heights[0], albedo_mode, shading_mode,
                              image_filter_size, texture_filter_size, compute_normal_map));
    hc_renderer_s* r = *out;
    r->ws.cam_w.assign(camera_widths, camera_widths + number_of_cameras);
    r->ws.cam_h.assign(camera_heights, camera_heights + number_of_cameras);
    return HC_OK;
}

extern "C" hc_status hc_renderer_frame_pixels(hc_renderer h, int64_t* pixels) {
    clear_error();
    HC_REQUIRE(h && pixels, "invalid arguments");
    *pixels = frame_pixels(h);
    return HC_OK;
}
