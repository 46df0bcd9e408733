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
/* Number of kernel launches this library has issued in this process
 * (launches recorded into a CUDA graph count once, at capture). */
int64_t hc_kernel_launches(void);

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
/* hc_renderer_create with one resolution per camera (camera_widths /
 * camera_heights [C], host; no reference counterpart: the reference op has
 * one render_resolution_u/v).  Views of different sizes are rasterised in
 * one launch.  Every per-pixel buffer of a call is then [B, P, ...] with P
 * the pixels of a frame (hc_renderer_frame_pixels), the frame's cameras
 * concatenated in order, each row-major H_c x W_c. */
hc_status hc_renderer_create_multires(hc_renderer* out, const int32_t* faces, int32_t n_faces,
                                      const float* texture_coordinates, int32_t n_texcoords,
                                      int32_t number_of_vertices, int32_t number_of_cameras,
                                      const int32_t* camera_widths, const int32_t* camera_heights,
                                      const char* albedo_mode, const char* shading_mode,
                                      int32_t image_filter_size, int32_t texture_filter_size,
                                      const char* compute_normal_map);
/* pixels of one frame (sum over cameras of W_c * H_c) */
hc_status hc_renderer_frame_pixels(hc_renderer h, int64_t* pixels);
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
 * Adjoint of the forward render (CudaRendererGradGpu).
 * Replaces CudaRendererGrad::Compute
 * (CudaRenderer/cpp/src/TensorflowOperators/CudaRenderer/CudaRendererGrad.cpp:6-34,241-274)
 * and renderBuffersGradGPU (CudaRenderer/cpp/src/Renderer/CUDABasedRasterizationGrad.cu:503-514).
 * Inputs in the op's order: render_buffer_grad [B,C,H,W,3], vertex_pos,
 * vertex_color, texture, sh_coeff, target_image [B,C,H,W,3], vertex_normal
 * [B,C,N,3], barycentric_buffer, face_buffer (the forward's saved outputs),
 * extrinsics, intrinsics.  Outputs (overwritten): vertex_pos_grad [B,N,3],
 * vertex_color_grad [B,N,3], texture_grad [B,TH,TW,3], sh_coeff_grad [B,C,27].
 * Only vertexColor and textured albedo carry gradients (the reference
 * registers zeros for the other modes, CudaRendererGPU.py:229-237).
 */
hc_status hc_renderer_backward(hc_renderer h, void* stream, int32_t batch,
                               const float* render_buffer_grad, const float* vertex_pos,
                               const float* vertex_color, const float* texture,
                               int32_t texture_height, int32_t texture_width, const float* sh_coeff,
                               const float* target_image, const float* vertex_normal,
                               const float* barycentric_buffer, const int32_t* face_buffer,
                               const float* extrinsics, const float* intrinsics,
                               float* vertex_pos_grad, float* vertex_color_grad, float* texture_grad,
                               float* sh_coeff_grad);

/*
 * The renderer with the training step's masked image L1 fused in (no
 * reference counterpart: the reference runs the L1 as separate TF ops,
 * HPCMeshDL.py:642-688, here hc_image_l1_loss).  hc_renderer_forward_l1
 * writes what hc_renderer_forward writes (compute_normal_map must be none)
 * and, from the pixels it shades, the L1 state (16 bytes, the layout of
 * hc_image_l1_loss's workspace: double sum of |255 R - 255 T|, uint64 count
 * of non-zero terms, over pixels with a face and a non-zero foreground_mask
 * [B,C,H,W] uint8, which may be NULL) and loss = sum / count (device float,
 * may be NULL).  hc_renderer_backward_l1 is hc_renderer_backward with the
 * image gradient 255 sign(255 R - 255 T) / count formed per pixel from
 * render_buffer, target_image and that state instead of read from a
 * gradient image.  Results equal hc_renderer_forward + hc_image_l1_loss +
 * hc_renderer_backward up to the summation order of the loss.
 */
hc_status hc_renderer_forward_l1(hc_renderer h, void* stream, int32_t batch, const float* vertex_pos,
                                 const float* vertex_color, const float* texture, int32_t texture_height,
                                 int32_t texture_width, const float* sh_coeff, const float* extrinsics,
                                 const float* intrinsics, float* barycentric_buffer, int32_t* face_buffer,
                                 float* render_buffer, float* vertex_normal, const float* target_image,
                                 const uint8_t* foreground_mask, void* l1_state, float* loss);
hc_status hc_renderer_backward_l1(hc_renderer h, void* stream, int32_t batch, const void* l1_state,
                                  const float* render_buffer, const uint8_t* foreground_mask,
                                  const float* vertex_pos, const float* vertex_color, const float* texture,
                                  int32_t texture_height, int32_t texture_width, const float* sh_coeff,
                                  const float* target_image, const float* vertex_normal,
                                  const float* barycentric_buffer, const int32_t* face_buffer,
                                  const float* extrinsics, const float* intrinsics, float* vertex_pos_grad,
                                  float* vertex_color_grad, float* texture_grad, float* sh_coeff_grad);

/*
 * Barycentric Jacobian of the adjoint.  0 (default): the exact derivative of
 * the ray-hit barycentrics in closed form (rank 1 per vertex); 1: the
 * reference's 3x9 formula (dJBCDVerpos, RendererUtil.h:670-861) evaluated as
 * written.  Both are the same function; they differ by float rounding, which
 * for the reference formula is ~1e-4 relative at millimetre scale.
 */
hc_status hc_renderer_set_gradient_parity(hc_renderer h, int32_t parity);

/*
 * Tile schedule of the adjoint's persistent CTAs (no reference counterpart).
 * 1 (default): the CTAs claim tiles from a counter, which balances tiles of
 * uneven cost; 0: CTA i takes tiles i, i + grid, ..., so CTAs that run out
 * early free their SM, which serves a caller that runs independent work on
 * another stream at the same time.  Results are the same either way.
 */
hc_status hc_renderer_set_adjoint_schedule(hc_renderer h, int32_t dynamic);

/*
 * Raster statistics of the last forward on this handle: triangle/tile pairs
 * binned and pairs that overflowed a tile bin and took the atomic spill path.
 * Synchronises `stream`; host output pointers, either may be NULL.
 */
hc_status hc_renderer_stats(hc_renderer h, void* stream, int64_t* binned, int64_t* spilled);

/* Per-kernel timing for benchmarks (no reference counterpart).  When enabled,
 * every renderer launch is bracketed by CUDA events on its stream;
 * hc_renderer_kernel_times writes the last recorded duration (ms) of each
 * kernel, in the order view set-up, vertex normals, triangle frames, binning,
 * spill, tile resolve, render adjoint, normal chain (-1 if not run since the
 * previous read), waiting for the last events.  Off by default; not for
 * stream capture. */
hc_status hc_renderer_set_kernel_timing(hc_renderer h, int32_t enable);
hc_status hc_renderer_kernel_times(hc_renderer h, float* ms, int32_t n);

/* ------------------------------------------------------------------------ */
/* Embedded-graph deformation                                                */
/* ------------------------------------------------------------------------ */

typedef struct hc_eg_s* hc_eg;

/*
 * Create an embedded graph over a base mesh (host arrays).  Replaces the
 * EmbeddedGraphGpu op construction (CustomTensorFlowCPPOperators/src/
 * CustomGPUOperators/EmbeddedGraphOperator/EmbeddedGraphGPUOp.cpp:6-25,30-120),
 * which reads the same arrays from the character / graph files
 * (Skeletool/Mesh/EmbeddedGraph.cpp:379-548): base vertices [N,3], faces
 * [F,3], node -> base-vertex index [M], the vertex -> node CSR (offsets,
 * sizes, indices, weights) and the node -> vertex CSR with the same weights,
 * optional markers [Mk,3] with their node [Mk].
 */
hc_status hc_eg_create(hc_eg* out, int32_t n_vertices, const float* base_vertices, const int32_t* faces,
                       int32_t n_faces, int32_t n_nodes, const int32_t* node_to_base_vertex,
                       const int32_t* v2n_offsets, const int32_t* v2n_sizes, const int32_t* v2n_indices,
                       const float* v2n_weights, const int32_t* n2v_offsets, const int32_t* n2v_sizes,
                       const int32_t* n2v_indices, const float* n2v_weights, int32_t n_markers,
                       const float* base_markers, const int32_t* marker_to_node);
hc_status hc_eg_destroy(hc_eg h);
hc_status hc_eg_reserve(hc_eg h, int32_t batch);
/* 0 (default): skinned-rotation/translation gradients are zero, as in the
 * reference (EmbeddedGraphGPUOpGrad.cu:136-142); 1: return them. */
hc_status hc_eg_set_full_skinned_gradient(hc_eg h, int32_t enable);

/*
 * Forward (EmbeddedGraphGpu; EmbeddedGraphGPUOp.cu:229-240).  Inputs
 * [B,M,3]: nodes_delta_translation, nodes_delta_rotation (Euler, rad),
 * nodes_skinned_translation, nodes_skinned_rotation; vertex_displacements
 * [B,N,3].  Outputs: deformed_vertices [B,N,3], deformed_normals [B,N,3]
 * (may be NULL), deformed_markers [B,Mk,3], deformed_graph [B,M,3] (may be
 * NULL), d_delta_rotation / d_skinned_rotation [B,M,3] (copies of the angle
 * inputs for the gradient op; may be NULL).
 */
hc_status hc_eg_forward(hc_eg h, void* stream, int32_t batch, const float* nodes_delta_translation,
                        const float* nodes_delta_rotation, const float* nodes_skinned_translation,
                        const float* nodes_skinned_rotation, const float* vertex_displacements,
                        float* deformed_vertices, float* deformed_normals, float* deformed_markers,
                        float* deformed_graph, float* d_delta_rotation, float* d_skinned_rotation);

/*
 * Adjoint (EmbeddedGraphGpuGrad; EmbeddedGraphGPUOpGrad.cu:204-213):
 * deformed_vertices_grad [B,N,3], deformed_markers_grad [B,Mk,3] (may be NULL),
 * d_delta_a / d_skinned_a [B,M,3] -> nodes_t_grad, nodes_r_grad,
 * nodes_skinned_t_grad, nodes_skinned_r_grad [B,M,3], vertex_displacements_grad
 * [B,N,3].  nodes_delta_translation and vertex_displacements (the forward
 * inputs) are only read with the full skinned gradient enabled (else NULL).
 */
hc_status hc_eg_backward(hc_eg h, void* stream, int32_t batch, const float* deformed_vertices_grad,
                         const float* deformed_markers_grad, const float* d_delta_a, const float* d_skinned_a,
                         float* nodes_t_grad, float* nodes_r_grad, float* nodes_skinned_t_grad,
                         float* nodes_skinned_r_grad, float* vertex_displacements_grad,
                         const float* nodes_delta_translation, const float* vertex_displacements);

/* ------------------------------------------------------------------------ */
/* Embedded-graph ARAP regulariser                                           */
/* ------------------------------------------------------------------------ */

typedef struct hc_arap_s* hc_arap;

/*
 * EmbeddedGraphArapGpu (EmbeddedGraphArapGPUOp.cpp:5-16, kernels
 * EmbeddedGraphArapGPUOp.cu:10-97).  The handle holds what the op's
 * constructor reads from the character and graph files
 * (EmbeddedGraphArapGPUOp.cpp:38-53): base vertices [N,3] (mm), node -> base
 * vertex [M], the node -> node CSR (offsets, sizes, indices; the graph mesh's
 * neighbours in ascending order, EmbeddedGraph.cpp:155-167, 420-436) and the
 * per-node rigidity weights [M] (EmbeddedGraph.cpp:460-490).
 * max_connections is the op attr max_number_of_node_connections (every node's
 * list must fit).
 */
hc_status hc_arap_create(hc_arap* out, int32_t n_vertices, const float* base_vertices, int32_t n_nodes,
                         const int32_t* node_to_base_vertex, const int32_t* n2n_offsets, const int32_t* n2n_sizes,
                         const int32_t* n2n_indices, const float* rigidity_weights, int32_t max_connections);
hc_status hc_arap_destroy(hc_arap h);
/*
 * nodes_translation, nodes_rotation (Euler, rad) [B,M,3] -> nodes_arap_loss
 * [B,M,max_connections,3] (R_j (g_k - g_j) + g_j + t_j - (g_k + t_k), zeros in
 * the padding slots), d_connection_weights [B,M,max_connections]
 * ((rho_j + rho_k) / 2, 0 in padding), d_rotation [B,M,3] (the rotation
 * input, for the gradient op).
 */
hc_status hc_arap_forward(hc_arap h, void* stream, int32_t batch, const float* nodes_translation,
                          const float* nodes_rotation, float* nodes_arap_loss, float* connection_weights,
                          float* rotation);
/*
 * EmbeddedGraphArapGpuGrad (EmbeddedGraphArapGPUOpGrad.cpp:5-15, kernel
 * EmbeddedGraphArapGPUOpGrad.cu:9-96): nodes_arap_loss gradient
 * [B,M,max_connections,3] and d_a [B,M,3] -> nodes_t_grad, nodes_r_grad
 * [B,M,3].  As the reference, the connection weights get no gradient and the
 * translation gradient of a pair takes the neighbour's slot that names this
 * node (the last one if it appears twice; none if it is missing).
 */
hc_status hc_arap_backward(hc_arap h, void* stream, int32_t batch, const float* nodes_arap_loss_grad,
                           const float* nodes_rotation, float* nodes_translation_grad, float* nodes_rotation_grad);

/* ------------------------------------------------------------------------ */
/* Forward kinematics + dual-quaternion / linear-blend skinning              */
/* ------------------------------------------------------------------------ */

typedef struct hc_skin_s* hc_skin;

/*
 * Create a skinned character from host arrays (what the reference reads from
 * its .character / .skeleton / .skin files, Skeletool/Character/
 * skinnedcharacter.cpp:425-559, skeleton.cpp).  Replaces the DqSkinningGpu /
 * LbSkinningGpu op construction (DQSkinningGPUOp.cpp:5-15,18-120;
 * LBSkinningGPUOp.cpp:5-16).
 *   joints: parent [J] (-1 = root, parents before children), joint_type [J]
 *   (0 revolute, 1 prismatic), offset [J,3] (local, mm), axis [J,3] (local
 *   unit axis), joint_scale [J] (NULL = 1);
 *   dofs: CSR dof_offsets [D+1] over (dof_joint, dof_weight) entries; a dof
 *   adds weight * value to each joint's parameter (dof.cpp:9-17);
 *   skinning joints: skin_joint [S] and skin_scale [S] (NULL = 1), whose
 *   transform is joint * scale * inverse(bind joint), the bind joint taken at
 *   zero dofs with every joint scale 1 (skeleton.cpp:2840-2853);
 *   mesh: base_vertices / base_normals [N,3], skin_index [N,K] (skinning joint
 *   per weight slot).
 */
hc_status hc_skin_create(hc_skin* out, int32_t n_joints, const int32_t* parent, const int32_t* joint_type,
                         const float* offset, const float* axis, const float* joint_scale, int32_t n_dofs,
                         const int32_t* dof_offsets, const int32_t* dof_joint, const float* dof_weight,
                         int32_t n_skin, const int32_t* skin_joint, const float* skin_scale, int32_t n_vertices,
                         const float* base_vertices, const float* base_normals, int32_t k,
                         const int32_t* skin_index);
hc_status hc_skin_destroy(hc_skin h);
hc_status hc_skin_reserve(hc_skin h, int32_t batch);
/* 1 (default): gradients reproduce the reference's formulas, including the
 * weight-Jacobian indexing slips (DQHelper.h:121-174,
 * LBSkinningGPUOpGrad.cu:22-32,65-74); 0: exact weight gradients. */
hc_status hc_skin_set_parity(hc_skin h, int32_t parity);

/* DqSkinningGpu forward (DQSkinningGPUOp.cpp:351-389 + DQSkinningGPUOp.cu:56-137),
 * forward kinematics on the device: dofs [B,D], skinning_weights [B,N,K] ->
 * skinned_vertex_positions / normals [B,N,3], global_joint_position /
 * axis [B,J,3], dual_quaternions [B,S,8] (rotation x,y,z,w then translation
 * x,y,z,w), output_skinning_weights [B,N,K] (copy; may be NULL). */
hc_status hc_dq_skinning_forward(hc_skin h, void* stream, int32_t batch, const float* dofs,
                                 const float* skinning_weights, float* skinned_vertex_positions,
                                 float* skinned_vertex_normals, float* global_joint_position,
                                 float* global_joint_axis, float* dual_quaternions,
                                 float* output_skinning_weights);
/* DqSkinningGpuGrad (DQSkinningGPUOpGrad.cu:12-217): dofs_grad [B,D] (the
 * reference's linearised rotation-about-axis derivative), skinning_weights_grad
 * [B,N,K]. */
hc_status hc_dq_skinning_backward(hc_skin h, void* stream, int32_t batch,
                                  const float* skinned_vertex_positions_grad,
                                  const float* skinned_vertex_positions, const float* global_joint_position,
                                  const float* global_joint_axis, const float* dual_quaternions,
                                  const float* skinning_weights, float* dofs_grad, float* skinning_weights_grad);
/* LbSkinningGpu forward (LBSkinningGPUOp.cu:49-113): + displacement [B,N,3];
 * transformation [B,S,12] (rotation row-major 9, translation 3). */
hc_status hc_lb_skinning_forward(hc_skin h, void* stream, int32_t batch, const float* dofs,
                                 const float* skinning_weights, const float* displacement,
                                 float* skinned_vertex_positions, float* skinned_vertex_normals,
                                 float* global_joint_position, float* global_joint_axis, float* transformation,
                                 float* output_skinning_weights);
/* LbSkinningGpuGrad (LBSkinningGPUOpGrad.cu:11-168): dofs_grad [B,D],
 * skinning_weights_grad [B,N,K], displacement_grad [B,N,3].  displacement is
 * only read in the exact mode (parity 0). */
hc_status hc_lb_skinning_backward(hc_skin h, void* stream, int32_t batch,
                                  const float* skinned_vertex_positions_grad,
                                  const float* skinned_vertex_positions, const float* global_joint_position,
                                  const float* global_joint_axis, const float* transformation,
                                  const float* skinning_weights, const float* displacement, float* dofs_grad,
                                  float* skinning_weights_grad, float* displacement_grad);

/* Pose2EmbeddedGraphCpu on the device (Pose2EmbeddedGraphCPUOp.cpp:6-13,129-300):
 * dofs [B,D] -> per embedded-graph node the blended dual quaternion of its
 * base vertex (node_vertex [M], device), with the character's skin weights
 * vertex_weights [N,K] (device), as nodes_skinned_translation [B,M,3] and
 * Z-Y-X Euler nodes_skinned_rotation [B,M,3] (the EG op's skinned inputs);
 * dual_quaternions [B,S,8] receives the skinning joints' dual quaternions. */
hc_status hc_pose2eg_forward(hc_skin h, void* stream, int32_t batch, const float* dofs, int32_t n_nodes,
                             const int32_t* node_vertex, const float* vertex_weights,
                             float* nodes_skinned_translation, float* nodes_skinned_rotation,
                             float* dual_quaternions);
/* Adjoint of hc_pose2eg_forward (no counterpart in the reference, which
 * registers no gradient for Pose2EmbeddedGraphCpu, Pose2EmbeddedGraphCpu.py:
 * 55-60): gradients of nodes_skinned_translation / nodes_skinned_rotation
 * [B,M,3] -> dofs_grad [B,D], exact through the Euler angles, the blended
 * dual quaternions and the kinematic chain.  Recomputes the forward
 * kinematics from dofs. */
hc_status hc_pose2eg_backward(hc_skin h, void* stream, int32_t batch, const float* dofs, int32_t n_nodes,
                              const int32_t* node_vertex, const float* vertex_weights,
                              const float* nodes_skinned_translation_grad,
                              const float* nodes_skinned_rotation_grad, float* dofs_grad);

/* ------------------------------------------------------------------------ */
/* Camera projection, projected-mesh boundary, silhouette DT loss            */
/* ------------------------------------------------------------------------ */

/* CameraProjectionGpu (CameraProjectionGPUOp.cu:12-102): points [B,N,3] (and
 * vectors [B,N,3] when is_point = 0), extrinsics [B,C*12], intrinsics [B,C*9]
 * -> points_image_space [B,C,N,2] (image points, or unit image-space
 * directions of the vectors). */
hc_status hc_camera_projection_forward(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                       const float* points_global_space, const float* vectors_global_space,
                                       const float* extrinsics, const float* intrinsics, int32_t is_point,
                                       float* points_image_space);
/* CameraProjectionGpuGrad (CameraProjectionGPUOpGrad.cu:12-111): [B,C,N,2]
 * gradient -> points_global_space_grad [B,N,3] (zero in vector mode, as the
 * reference registers for normals). */
hc_status hc_camera_projection_backward(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                        const float* points_image_space_grad, const float* points_global_space,
                                        const float* extrinsics, const float* intrinsics, int32_t is_point,
                                        float* points_global_space_grad);
typedef struct hc_mesh_boundary_s* hc_mesh_boundary;

/* ProjectedMeshBoundaryGpu (ProjectedMeshBoundaryGPUOp.cpp:5-17,139-160;
 * Skeletool/Mesh/CUDABasedRasterization.cu:53-206).  The handle holds the
 * mesh faces (the op's mesh_file_path_boundary_check).  Forward projects
 * points_global_space [B,N,3] with extrinsics [B,12C] / intrinsics [B,9C]
 * (or takes the projection from points_image_space [B,C,N,2] when that is
 * non-NULL: CameraProjectionGpu gives the identical points), rasterises the
 * image-space coverage of the mesh at width x height (render_u x render_v)
 * and flags a vertex of a view when a pixel of the 3x3 window around its
 * truncated projection is uncovered.  is_boundary [B,C,N] uint8 (TF bool).
 * width and height lie in [3, 32767].  Bit-identical to the reference op. */
hc_status hc_mesh_boundary_create(hc_mesh_boundary* out, const int32_t* faces, int32_t n_faces,
                                  int32_t n_vertices);
hc_status hc_mesh_boundary_destroy(hc_mesh_boundary h);
hc_status hc_mesh_boundary_reserve(hc_mesh_boundary h, int32_t batch, int32_t n_cameras, int32_t width,
                                   int32_t height);
hc_status hc_mesh_boundary_forward(hc_mesh_boundary h, void* stream, int32_t batch, int32_t n_cameras,
                                   int32_t width, int32_t height, const float* points_global_space,
                                   const float* extrinsics, const float* intrinsics,
                                   const float* points_image_space, uint8_t* is_boundary);
/* hc_mesh_boundary_forward with a per-pixel face hint: face_hint [B,C,H,W]
 * int32, e.g. the face buffer of hc_renderer_forward for the same vertices,
 * cameras and resolution.  A vertex's flag reads the 3x3 pixel window around
 * its projection; a window pixel whose hint face passes the op's own 2-D
 * coverage test (checked exactly) is covered, and only the other pixels of
 * those windows, with the tiles that hold them, go through the full binned
 * coverage.  The flags are
 * bit-identical to hc_mesh_boundary_forward for every hint (out-of-range ids
 * count as no hint); a hint that matches the coverage only saves work.  No
 * reference counterpart (the reference op rasterises the whole mesh again). */
hc_status hc_mesh_boundary_forward_hinted(hc_mesh_boundary h, void* stream, int32_t batch, int32_t n_cameras,
                                          int32_t width, int32_t height, const float* points_global_space,
                                          const float* extrinsics, const float* intrinsics,
                                          const float* points_image_space, const int32_t* face_hint,
                                          uint8_t* is_boundary);
/* hc_mesh_boundary_forward for cameras of different image sizes (no
 * reference counterpart: the reference needs one op instance per resolution).
 * widths / heights: host arrays [C]; per-pixel data of a frame are its
 * cameras' images concatenated in camera order (row-major H_c x W_c), as for
 * hc_renderer_create_multires.  face_hint [B, pixels of a frame] int32 or
 * NULL (then as hc_mesh_boundary_forward).  Cameras of one size behave as
 * hc_mesh_boundary_forward(_hinted); mixed sizes take at most 32 cameras per
 * call.  Each camera's flags are those of the single-size op at its size. */
hc_status hc_mesh_boundary_reserve_sized(hc_mesh_boundary h, int32_t batch, int32_t n_cameras,
                                         const int32_t* widths, const int32_t* heights);
hc_status hc_mesh_boundary_forward_sized(hc_mesh_boundary h, void* stream, int32_t batch, int32_t n_cameras,
                                         const int32_t* widths, const int32_t* heights,
                                         const float* points_global_space, const float* extrinsics,
                                         const float* intrinsics, const float* points_image_space,
                                         const int32_t* face_hint, uint8_t* is_boundary);
/* The same boundary test with coverage taken from a renderer face buffer
 * [B,C,H,W] (-1 = empty) instead of the op's own 2-D raster.  No separate
 * reference counterpart: the renderer's ray test and the 2-D barycentric test
 * disagree on some pixels along triangle edges, so flags can differ from
 * ProjectedMeshBoundaryGpu there.  is_boundary [B,C,N] uint8. */
hc_status hc_projected_mesh_boundary(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                     int32_t width, int32_t height, const float* points_image_space,
                                     const int32_t* face_buffer, uint8_t* is_boundary);

typedef struct hc_silhouette_s* hc_silhouette;
hc_status hc_silhouette_create(hc_silhouette* out);
hc_status hc_silhouette_destroy(hc_silhouette h);
hc_status hc_silhouette_reserve(hc_silhouette h, int32_t batch, int32_t n_cameras, int32_t n_points,
                                int32_t resolution_u, int32_t resolution_v);
/*
 * MultiViewSilhouetteLossGpu (MultiViewSilhouetteLossGPUOp.cu:11-251):
 * points / normals_image_space [B,C,N,2], is_boundary [B,C,N] uint8,
 * distance_transform_image [B,C,U,V] uint8 stored with rows of U values (the
 * reference's indexing), multi_view_crops [B,C,7] -> mv_dt_residual [B,C,N],
 * mv_dt_residual_1 [B,C,V,U,2], dt_image_gradient [B,C,N,2],
 * closest_vertex_id [B,C,V,U] (float, -1 = none).
 */
hc_status hc_silhouette_forward(hc_silhouette h, void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                int32_t resolution_u, int32_t resolution_v, const float* points_image_space,
                                const float* normals_image_space, const uint8_t* is_boundary,
                                const uint8_t* distance_transform_image, const float* multi_view_crops,
                                float* mv_dt_residual, float* mv_dt_residual_1, float* dt_image_gradient,
                                float* closest_vertex_id);
/* MultiViewSilhouetteLossGpuGrad (MultiViewSilhouetteLossGPUOpGrad.cu:11-72)
 * -> points_image_space_grad [B,C,N,2] (overwritten). */
hc_status hc_silhouette_backward(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                 int32_t resolution_u, int32_t resolution_v, const float* mv_dt_grad,
                                 const float* mv_dt_grad_1, const float* dt_image_grad,
                                 const float* closest_vertex_id, const float* multi_view_crops,
                                 float* points_image_space_grad);

/* The silhouette loss and its adjoint for cameras of different image sizes
 * (no reference counterpart: the reference needs one op instance per
 * resolution).  widths (U) / heights (V): host arrays [C]; the distance
 * images and the per-pixel outputs hold a frame's cameras concatenated in
 * camera order, each row-major V_c x U_c: distance_transform_image
 * [B, pixels of a frame] uint8, mv_dt_residual_1 [B, pixels of a frame, 2],
 * closest_vertex_id [B, pixels of a frame].  Cameras of one size behave as
 * hc_silhouette_forward / _backward; mixed sizes take at most 32 cameras per
 * call.  Each camera's results are those of the single-size op at its size. */
hc_status hc_silhouette_reserve_sized(hc_silhouette h, int32_t batch, int32_t n_cameras, int32_t n_points,
                                      const int32_t* widths, const int32_t* heights);
hc_status hc_silhouette_forward_sized(hc_silhouette h, void* stream, int32_t batch, int32_t n_cameras,
                                      int32_t n_points, const int32_t* widths, const int32_t* heights,
                                      const float* points_image_space, const float* normals_image_space,
                                      const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                                      const float* multi_view_crops, float* mv_dt_residual, float* mv_dt_residual_1,
                                      float* dt_image_gradient, float* closest_vertex_id);
hc_status hc_silhouette_backward_sized(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                       const int32_t* widths, const int32_t* heights, const float* mv_dt_grad,
                                       const float* mv_dt_grad_1, const float* dt_image_grad,
                                       const float* closest_vertex_id, const float* multi_view_crops,
                                       float* points_image_space_grad);

/* The silhouette loss with the squared loss of its per-pixel residual fused
 * in (no reference counterpart; the reference graph squares and sums the
 * residual image with TF ops, HPCMeshDL.py:669-688).
 * hc_silhouette_forward_sumsq_sized is hc_silhouette_forward_sized that also
 * forms sum(mv_dt_residual_1^2) while it writes the residual, into *sumsq_1
 * (a device double, cleared by the call), and writes the loss
 * weight_1 * sum into *loss_1 (a device float).  Only pixels on the target's
 * silhouette have a non-zero residual, so no pass over the residual image
 * follows.  hc_silhouette_backward_scaled_sized is
 * hc_silhouette_backward_sized with the residual's upstream gradient given as
 * scale_1 x mv_dt_grad_1: passing the residual itself and scale_1 = 2 weight_1
 * gives the squared loss's adjoint without a dense gradient image (the same
 * values as forming 2 w x residual first: the product is rounded once either
 * way). */
hc_status hc_silhouette_forward_sumsq_sized(hc_silhouette h, void* stream, int32_t batch, int32_t n_cameras,
                                            int32_t n_points, const int32_t* widths, const int32_t* heights,
                                            const float* points_image_space, const float* normals_image_space,
                                            const uint8_t* is_boundary, const uint8_t* distance_transform_image,
                                            const float* multi_view_crops, float* mv_dt_residual,
                                            float* mv_dt_residual_1, float* dt_image_gradient,
                                            float* closest_vertex_id, float weight_1, double* sumsq_1,
                                            float* loss_1);
hc_status hc_silhouette_backward_scaled_sized(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                              const int32_t* widths, const int32_t* heights,
                                              const float* mv_dt_grad, const float* mv_dt_grad_1, float scale_1,
                                              const float* dt_image_grad, const float* closest_vertex_id,
                                              const float* multi_view_crops, float* points_image_space_grad);

/*
 * hc_silhouette_forward without allocation.  No counterpart in the reference.
 * For callers that cannot allocate device memory themselves: a TensorFlow
 * custom op must take its memory from TF's allocator, and hosts that reserve
 * everything at start-up forbid cudaMalloc on their hot path.  Same arguments
 * and results as hc_silhouette_forward minus the handle: the boundary-vertex
 * grid lives in a fixed 8 MiB device array inside the library (held by every
 * GPU that loads it, until the process exits), which limits a call to
 *   4 * (B*C * (3 * (ceil(U/30)+3) * (ceil(V/30)+3) + N) + 1) <= 8 MiB,
 * e.g. 8 views of 1024x1024 with N = 40,962; larger calls return
 * HC_ERR_INVALID.  The first call on a device resolves the array's device
 * address with that device current; make that first call before any stream
 * capture begins.  All calls on a device share the one array and it keeps the last call's contents: calls
 * whose kernels overlap on the GPU (e.g. issued on different streams) race,
 * so order them on one stream.
 */
hc_status hc_silhouette_forward_static(void* stream, int32_t batch, int32_t n_cameras, int32_t n_points,
                                       int32_t resolution_u, int32_t resolution_v, const float* points_image_space,
                                       const float* normals_image_space, const uint8_t* is_boundary,
                                       const uint8_t* distance_transform_image, const float* multi_view_crops,
                                       float* mv_dt_residual, float* mv_dt_residual_1, float* dt_image_gradient,
                                       float* closest_vertex_id);

/* ------------------------------------------------------------------------ */
/* Losses                                                                    */
/* ------------------------------------------------------------------------ */

/*
 * Masked L1 image loss of the training step and its gradient.
 * Replaces the TF graph of Projects/HoloportedCharacters/HPCMeshDL.py:669-688:
 * difference = 255 (render - target) * mask * (face >= 0),
 * loss = sum |difference| / count_nonzero(difference),
 * render_buffer_grad = 255 sign(difference) * mask * (face >= 0) / count.
 * n_pixels = B*C*H*W; render/target are [n_pixels,3]; face_buffer [n_pixels];
 * foreground_mask [n_pixels] uint8 (NULL = all ones); loss is one device
 * float; workspace is device scratch of at least 16 bytes (its contents on
 * entry are ignored).
 */
hc_status hc_image_l1_loss(void* stream, int64_t n_pixels, const float* render_buffer,
                           const float* target_image, const int32_t* face_buffer,
                           const uint8_t* foreground_mask, void* workspace, float* loss,
                           float* render_buffer_grad);

/*
 * Sum-of-squares loss of a residual and its gradient: loss = weight * sum x^2,
 * grad = 2 * weight * x (n floats).  The silhouette residuals of
 * MultiViewSilhouetteLossGpu (mv_dt_residual, mv_dt_residual_1) are trained
 * with it; the reference leaves this reduction to the TF graph.  workspace is
 * device scratch of at least 8 bytes.
 */
hc_status hc_sum_squares_loss(void* stream, int64_t n, const float* x, float weight, void* workspace, float* loss,
                              float* grad);

/*
 * Gaussian smoothing of target images (GaussianSmoothingGpu.smoothImage,
 * Projects/CustomTFOperators/GaussianSmoothingGpu.py:12-37): image [n, H, W,
 * channels] (channels <= 4) convolved per channel with the (2 size + 1)^2
 * normalised Gaussian of the given mean / std, zero padding; size <= 15.
 * size == 0 or std == 0 copies the image, as the reference returns it.
 */
hc_status hc_gaussian_smooth(void* stream, int32_t n_images, int32_t height, int32_t width, int32_t channels,
                             int32_t size, float mean, float std, const float* image, float* out);

/* dst += src over n floats: the AddN that TF inserts where two gradient
 * branches meet on one tensor (e.g. vertex positions, fed by the renderer
 * and by the silhouette's camera projection). */
hc_status hc_add_inplace(void* stream, int64_t n, float* dst, const float* src);

/* dst[i] = src[i] / 255 (float32, IEEE division) over n values: 8-bit target
 * images uploaded as bytes and widened on the device, a quarter of the
 * host-to-device traffic of float32 images.  src 4-byte and dst 16-byte
 * aligned.  No reference counterpart. */
hc_status hc_image_u8_to_f32(void* stream, int64_t n, const uint8_t* src, float* dst);

#ifdef __cplusplus
}
#endif

#endif /* HC_H_ */
