/*
 * CPU restatement of the reference deform-and-render chain -- TEST ORACLE.
 *
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg load
 * this library; the product never does.  Every function follows the
 * reference lines cited next to it.  Each one exists in two precisions:
 * the _f64 variant is the FP64 oracle used for error reports and finite
 * differences, the _f32 variant is the reference arithmetic in float on the
 * host cores (the CPU baseline).
 *
 * Parity pinning: the reference ships no tests, golden vectors or fixtures
 * for this path; its own CUDA kernels, compiled unmodified from the reference
 * tree (oracle/_ref), are the second oracle, run on the GPU, and the golden
 * files under tests/golden were produced by them.
 */
#ifndef HC_ORACLE_H_
#define HC_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Renderer forward (CUDABasedRasterization.cu:23-451 + renderBuffersGPU :553-576).
 * Shapes as in include/hc.h.  Extra per-pixel outputs (may be NULL):
 *   depth_q   [B,C,H,W] quantised depth int(t*1e4) of the winner, INT32_MAX if empty
 *   tie_count [B,C,H,W] triangles reaching the winner's quantised depth
 *   fragile   [B,C,H,W] 1 where a decision is within rounding of flipping:
 *             a candidate within 1e-5 (relative) of an edge, or two candidates
 *             within one depth quantum, or the winner's t*1e4 within 1e-3 of
 *             an integer (only computed by the f64 variant).
 * Winner among equal quantised depths: smallest face id.
 * nthreads <= 0 uses all OpenMP threads. */
int hco_render_forward_f64(int N, int F, const int32_t* faces, const float* texcoords, int B, int C, int W, int H,
                           int albedo, int shading, const float* verts, const float* colors, const float* texture,
                           int TH, int TW, const float* sh, const float* extr, const float* intr, float* bary,
                           int32_t* face, float* render, float* vnormal, int32_t* depth_q, int32_t* tie_count,
                           uint8_t* fragile, int nthreads);
int hco_render_forward_f32(int N, int F, const int32_t* faces, const float* texcoords, int B, int C, int W, int H,
                           int albedo, int shading, const float* verts, const float* colors, const float* texture,
                           int TH, int TW, const float* sh, const float* extr, const float* intr, float* bary,
                           int32_t* face, float* render, float* vnormal, int32_t* depth_q, int32_t* tie_count,
                           uint8_t* fragile, int nthreads);

/* Renderer adjoint (CUDABasedRasterizationGrad.cu:114-514), shapes as
 * hc_renderer_backward in include/hc.h; outputs are overwritten. */
int hco_render_backward_f64(int N, int F, const int32_t* faces, const float* texcoords, int B, int C, int W, int H,
                            int albedo, int shading, int ifs, int tfs, const float* grad, const float* verts,
                            const float* colors, const float* texture, int TH, int TW, const float* sh,
                            const float* target, const float* vnormal, const float* bary, const int32_t* face,
                            const float* extr, const float* intr, float* vpos_grad, float* vcol_grad,
                            float* tex_grad, float* sh_grad, int nthreads);
int hco_render_backward_f32(int N, int F, const int32_t* faces, const float* texcoords, int B, int C, int W, int H,
                            int albedo, int shading, int ifs, int tfs, const float* grad, const float* verts,
                            const float* colors, const float* texture, int TH, int TW, const float* sh,
                            const float* target, const float* vnormal, const float* bary, const int32_t* face,
                            const float* extr, const float* intr, float* vpos_grad, float* vcol_grad,
                            float* tex_grad, float* sh_grad, int nthreads);

/* Embedded-graph forward / adjoint (EmbeddedGraphGPUOp.cu:11-225,
 * EmbeddedGraphGPUOpGrad.cu:9-201); full = 1 adds the skinned gradients. */
#define HCO_EG_DECL(P)                                                                                          \
    int hco_eg_forward_##P(int B, int N, int M, int Mk, int F, const float* base, const int32_t* faces,        \
                           const int32_t* node_vertex, const int32_t* v2n_off, const int32_t* v2n_size,         \
                           const int32_t* v2n_idx, const float* v2n_w, const float* markers, const int32_t* m2n, \
                           const float* dT, const float* dA, const float* sT, const float* sA, const float* disp, \
                           float* out_v, float* out_n, float* out_m, float* out_g);                              \
    int hco_eg_backward_##P(int B, int N, int M, int Mk, const float* base, const int32_t* node_vertex,        \
                            const int32_t* v2n_off, const int32_t* v2n_size, const int32_t* v2n_idx,           \
                            const float* v2n_w, const int32_t* n2v_off, const int32_t* n2v_size,                \
                            const int32_t* n2v_idx, const float* n2v_w, const int32_t* n2m, const float* markers, \
                            const float* gv, const float* gm, const float* dT, const float* dA, const float* sA, \
                            const float* disp, int full, float* gT, float* gA, float* gsT, float* gsA, float* gdisp);
HCO_EG_DECL(f64)
HCO_EG_DECL(f32)
/* FP64 forward with double outputs (finite differences) */
int hco_eg_forward_f64d(int B, int N, int M, int Mk, int F, const float* base, const int32_t* faces,
                        const int32_t* node_vertex, const int32_t* v2n_off, const int32_t* v2n_size,
                        const int32_t* v2n_idx, const float* v2n_w, const float* markers, const int32_t* m2n,
                        const float* dT, const float* dA, const float* sT, const float* sA, const float* disp,
                        double* out_v, double* out_n, double* out_m, double* out_g);


/* The reference's host kinematics in float (Skeletool joint / dof / skeleton
 * update with the dual-quaternion joint chain, DQSkinningGPUOp.cpp:257-347;
 * see hc_oracle_fk.inc): dofs [B,D] -> global joint positions / axes [B,J,3]
 * and the skinning joints' dual quaternions [B,S,8] (x, y, z, w rotation, then
 * x, y, z, w translation).  joint_scale / skin_scale may be NULL (ones). */
int hco_fk_f32(int B, int J, const int32_t* parent, const int32_t* type, const float* offset, const float* axis,
               const float* joint_scale, int D, const int32_t* dof_offsets, const int32_t* dof_joint,
               const float* dof_weight, int S, const int32_t* skin_joint, const float* skin_scale,
               const float* dofs, float* joint_position, float* joint_axis, float* dual_quaternions);
/* Pose2EmbeddedGraphCpu's node loop (Pose2EmbeddedGraphCPUOp.cpp:196-290) in
 * float on given joint dual quaternions [B,S,8]: skin_index / skin_weight
 * [N,K], node_vertex [M] -> skinned_t, skinned_a (Z-Y-X Euler) [B,M,3]. */
int hco_pose2eg_f32(int B, int S, int N, int K, const int32_t* skin_index, const float* skin_weight, int M,
                    const int32_t* node_vertex, const float* dual_quaternions, float* skinned_t, float* skinned_a);

#ifdef __cplusplus
}
#endif

#endif
