/*
 * hc.h -- C ABI of the B200 deform-and-render chain (libhc.so).
 *
 * Every entry point takes plain pointers and sizes, never a framework tensor
 * type, so TensorFlow custom ops, torch extensions, ctypes or any other FFI
 * can bind it.  All tensor arguments are caller-owned DEVICE pointers to
 * dense row-major float32 / int32 arrays with the shapes and layouts of the
 * reference ops they replace; host pointers are marked "host".
 *
 * Conventions
 *  - Every call returns an hc_status (0 = success) and never exits the
 *    process; hc_last_error() gives a message for the calling thread.
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *    default stream.  Calls enqueue work and do not synchronise the host, so
 *    a forward/backward sequence can be captured in a CUDA graph once the
 *    handle's workspace is reserved (hc_*_reserve) for the largest batch.
 *  - A handle owns its topology and scratch workspace; calls on one handle
 *    must be ordered (one stream, or serialised by the caller).  Independent
 *    handles may run concurrently.
 */
#ifndef HC_H_
#define HC_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t hc_status;
enum {
    HC_OK = 0,
    HC_ERR_INVALID = 1,   /* bad argument, shape or mode */
    HC_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    HC_ERR_ALLOC = 3,     /* device allocation failed */
    HC_ERR_OVERFLOW = 4,  /* a fixed-capacity work list overflowed; result incomplete */
    HC_ERR_TIMEOUT = 5    /* a bounded device wait gave up */
};

/* Message of the last failing call on this thread ("" if none). */
const char* hc_last_error(void);
/* Library version string. */
const char* hc_version(void);

/* ------------------------------------------------------------------------ */
/* Rasterizer / renderer                                                     */
/* ------------------------------------------------------------------------ */

typedef struct hc_renderer_s* hc_renderer;

/*
 * Create a renderer for a fixed topology and camera rig.
 * Replaces the CudaRendererGpu / CudaRendererGradGpu op construction
 * (CudaRenderer/cpp/src/TensorflowOperators/CudaRenderer/CudaRenderer.cpp:5-31,35-181;
 *  CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cpp:11-135) with the
 * same attributes: faces (host, int32[3F]), texture_coordinates (host,
 * float[6F] per face corner, may be NULL when n_texcoords == 0),
 * number_of_vertices, number_of_cameras, render_resolution_u (width),
 * render_resolution_v (height), albedo_mode ("vertexColor", "textured",
 * "normal", "lighting", "foregroundMask", "position", "depth", "uv"),
 * shading_mode ("shaded", "shadeless"; forced to "shadeless" for the modes
 * other than vertexColor and textured, as the reference op does),
 * image_filter_size, texture_filter_size, compute_normal_map ("none",
 * "normal", "position", "face").
 */
hc_status hc_renderer_create(hc_renderer* out, const int32_t* faces, int32_t n_faces,
                             const float* texture_coordinates, int32_t n_texcoords,
                             int32_t number_of_vertices, int32_t number_of_cameras,
                             int32_t render_resolution_u, int32_t render_resolution_v,
                             const char* albedo_mode, const char* shading_mode,
                             int32_t image_filter_size, int32_t texture_filter_size,
                             const char* compute_normal_map);
hc_status hc_renderer_destroy(hc_renderer h);

/* Pre-size the workspace for up to `batch` frames (no allocation afterwards). */
hc_status hc_renderer_reserve(hc_renderer h, int32_t batch);

/* Raster tuning: screen tile edge in pixels (8, 16 or 32) and per-tile bin
 * capacity; triangles beyond the capacity of a tile take the 64-bit atomicMin
 * spill path.  Defaults: 16 and 512. */
hc_status hc_renderer_set_tuning(hc_renderer h, int32_t tile, int32_t bin_capacity);

/*
 * Forward render of `batch` frames x C views.
 * Replaces CudaRendererGpu::Compute (CudaRenderer.cpp:316-345) and
 * renderBuffersGPU (CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cu:553-576).
 * Inputs: vertex_pos [B,N,3], vertex_color [B,N,3], texture [B,TH,TW,3],
 * sh_coeff [B,C,27], extrinsics [B,C*12] (row-major 3x4 world->camera),
 * intrinsics [B,C*9] (row-major 3x3).  Outputs: barycentric_buffer [B,C,H,W,2],
 * face_buffer [B,C,H,W] (int32, -1 = background), render_buffer [B,C,H,W,3],
 * vertex_normal [B,C,N,3], normal_map [B,TH,TW,3] (may be NULL when
 * compute_normal_map is "none").  texture may be NULL for modes that do not
 * sample it.
 */
hc_status hc_renderer_forward(hc_renderer h, void* stream, int32_t batch,
                              const float* vertex_pos, const float* vertex_color,
                              const float* texture, int32_t texture_height, int32_t texture_width,
                              const float* sh_coeff, const float* extrinsics, const float* intrinsics,
                              float* barycentric_buffer, int32_t* face_buffer, float* render_buffer,
                              float* vertex_normal, float* normal_map);

/*
 * hc_renderer_forward plus per-pixel diagnostics: depth_q [B,C,H,W] int32 is
 * the quantised depth int(t*1e4) of the visible triangle (INT32_MAX for
 * background; the reference's internal depth buffer,
 * CUDABasedRasterization.cu:241-251) and tie_count [B,C,H,W] int32 is the
 * number of triangles that reached that same quantised depth (>= 2 marks a
 * depth tie, where the reference's winner is arbitrary).  Either may be NULL.
 */
hc_status hc_renderer_forward_ex(hc_renderer h, void* stream, int32_t batch,
                                 const float* vertex_pos, const float* vertex_color,
                                 const float* texture, int32_t texture_height, int32_t texture_width,
                                 const float* sh_coeff, const float* extrinsics, const float* intrinsics,
                                 float* barycentric_buffer, int32_t* face_buffer, float* render_buffer,
                                 float* vertex_normal, float* normal_map,
                                 int32_t* depth_q, int32_t* tie_count);

/*
 * Raster statistics of the last forward on this handle: triangle/tile pairs
 * binned and pairs that overflowed a tile bin and took the atomic spill path.
 * Synchronises `stream`; host output pointers, either may be NULL.
 */
hc_status hc_renderer_stats(hc_renderer h, void* stream, int64_t* binned, int64_t* spilled);

#ifdef __cplusplus
}
#endif

#endif /* HC_H_ */
