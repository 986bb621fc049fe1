/*
 * sbh_b200 -- XLA custom-call (FFI) handlers of libsbh_b200.so.
 *
 * Same symbol names, argument order, result order and attribute names as
 * the reference's handlers (bhorowitz/barnes-hut src/sbh_ffi.cu, the
 * XLA_FFI_DEFINE_HANDLER_SYMBOL block at :3580-3947), so the reference's
 * python/jax_sbh_ffi.py (:44-338) can load this library and register every
 * target unchanged:
 *     jax.ffi.register_ffi_target(name, jax.ffi.pycapsule(lib.<symbol>),
 *                                 platform="CUDA", api_version=1)
 * Each handler takes XLA's call frame (XLA FFI C ABI, API version 0.1),
 * answers XLA's metadata query at registration, decodes its buffers and
 * scalar attributes (by name), takes the stream from the execution context
 * and calls the matching C entry point of sbh_b200.h. Scratch comes from
 * XLA's device allocator when the runtime offers one, else from
 * cudaMallocAsync on the same stream; nothing synchronises. Errors are
 * returned as XLA errors: INVALID_ARGUMENT with the reference's messages for
 * shape and size mismatches, INTERNAL for CUDA failures. Unlike the
 * reference, no parameter travels through __constant__ memory, so calls on
 * different streams do not race.
 */
#ifndef SBH_XLA_FFI_H_
#define SBH_XLA_FFI_H_

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct XLA_FFI_CallFrame XLA_FFI_CallFrame;
typedef struct XLA_FFI_Error XLA_FFI_Error;

/* direct sums: BruteForceGravity :548, SoftenedDirectForce :600, SoftenedDirectForceVjp :663 */
XLA_FFI_Error* sbh_bruteforce_gravity_ffi(XLA_FFI_CallFrame* call_frame);    /* :3580 */
XLA_FFI_Error* sbh_direct_force_soft_ffi(XLA_FFI_CallFrame* call_frame);     /* :3592 */
XLA_FFI_Error* sbh_direct_force_soft_vjp_ffi(XLA_FFI_CallFrame* call_frame); /* :3606 */

/* builds: BuildOctreeLevel3Buffers :736, BuildOctree8Buffers :1039 */
XLA_FFI_Error* sbh_build_octree_level3_buffers_ffi(XLA_FFI_CallFrame* call_frame); /* :3621 */
XLA_FFI_Error* sbh_build_octree8_buffers_ffi(XLA_FFI_CallFrame* call_frame);       /* :3634 */

/* Node2 / Node3 warp-vote BH: BarnesHutGravity{,3D} :2444,:2490, BarnesHutForce{,3D} :2563,:2729,
 * SoftenedBarnesHutForce{,3D} :2613,:2671 */
XLA_FFI_Error* sbh_barnes_hut_gravity_ffi(XLA_FFI_CallFrame* call_frame);       /* :3648 */
XLA_FFI_Error* sbh_barnes_hut_force_ffi(XLA_FFI_CallFrame* call_frame);         /* :3661 */
XLA_FFI_Error* sbh_barnes_hut_gravity_ffi_3d(XLA_FFI_CallFrame* call_frame);    /* :3674 */
XLA_FFI_Error* sbh_barnes_hut_force_ffi_3d(XLA_FFI_CallFrame* call_frame);      /* :3687 */
XLA_FFI_Error* sbh_barnes_hut_force_soft_ffi(XLA_FFI_CallFrame* call_frame);    /* :3750 */
XLA_FFI_Error* sbh_barnes_hut_force_soft_ffi_3d(XLA_FFI_CallFrame* call_frame); /* :3765 */

/* octree8 classic BH: BarnesHutForceOctree8 :3133, SoftenedBarnesHutForceOctree8 :3183,
 * SoftenedBarnesHutForceOctree8Vjp :3250 */
XLA_FFI_Error* sbh_barnes_hut_force_octree8_ffi(XLA_FFI_CallFrame* call_frame);          /* :3700 */
XLA_FFI_Error* sbh_barnes_hut_force_octree8_soft_ffi(XLA_FFI_CallFrame* call_frame);     /* :3713 */
XLA_FFI_Error* sbh_barnes_hut_force_octree8_soft_vjp_ffi(XLA_FFI_CallFrame* call_frame); /* :3731 */

/* Node2 / Node3 MLPCV: StochasticBarnesHut{Gravity,Force}{,3D} :2779-2944,
 * SoftenedStochasticBarnesHutForce{,3D} :2999,:3066 */
XLA_FFI_Error* sbh_stochastic_bh_gravity_ffi(XLA_FFI_CallFrame* call_frame);       /* :3780 */
XLA_FFI_Error* sbh_stochastic_bh_gravity_ffi_3d(XLA_FFI_CallFrame* call_frame);    /* :3795 */
XLA_FFI_Error* sbh_stochastic_bh_force_ffi(XLA_FFI_CallFrame* call_frame);         /* :3810 */
XLA_FFI_Error* sbh_stochastic_bh_force_ffi_3d(XLA_FFI_CallFrame* call_frame);      /* :3825 */
XLA_FFI_Error* sbh_stochastic_bh_force_soft_ffi(XLA_FFI_CallFrame* call_frame);    /* :3914 */
XLA_FFI_Error* sbh_stochastic_bh_force_soft_ffi_3d(XLA_FFI_CallFrame* call_frame); /* :3931 */

/* octree8 MLPCV: (Softened)StochasticBarnesHutForceOctree8{,Vjp} :3322,:3375,:3445,:3503 */
XLA_FFI_Error* sbh_stochastic_bh_force_octree8_ffi(XLA_FFI_CallFrame* call_frame);          /* :3840 */
XLA_FFI_Error* sbh_stochastic_bh_force_octree8_soft_ffi(XLA_FFI_CallFrame* call_frame);     /* :3856 */
XLA_FFI_Error* sbh_stochastic_bh_force_octree8_vjp_ffi(XLA_FFI_CallFrame* call_frame);      /* :3876 */
XLA_FFI_Error* sbh_stochastic_bh_force_octree8_soft_vjp_ffi(XLA_FFI_CallFrame* call_frame); /* :3893 */

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* SBH_XLA_FFI_H_ */
