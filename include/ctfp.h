/*
 * ctfp.h — C ABI of the B200 polyenergetic cone-beam forward projector.
 *
 * This is the device boundary that replaces the reference's GPU layer
 * (Source/CUDAFun/CBCTPolyProjGPU.cuh:33-114).  The reference exposed free
 * C++ functions taking its structs by value and kept process-global texture
 * state (CBCTPolyProjGPU.cu:8-10), reset the device in every init
 * (CBCTPolyProjGPU.cu:494) and printed-and-ignored CUDA errors
 * (CBCTPolyProjGPU.cu:55-61).  Here every call returns a ctfp_status, the
 * device is never reset, all state lives in a plan object, and the caller owns
 * every device buffer it passes in (volumes, outputs, checkpoints, gradients).
 *
 * Layouts (C order, last index fastest):
 *   volume      [pNumZ][pNumY][pNumX]  float32, one buffer per material
 *   projections [projNum][dNumV][dNumU] float32
 *   I0          [dNumV][dNumU]          float32
 *   L checkpoint[projNum][dNumV][dNumU][M] float32 (per-ray material path
 *               integrals, g/cm^3 * mm)
 *
 * Streams are passed as void* (a cudaStream_t; NULL = legacy default stream).
 * All launches are asynchronous on that stream; outputs are valid after the
 * stream is synchronised.  One plan may be used from one host thread at a time;
 * distinct plans are independent.
 */
#ifndef CTFP_H
#define CTFP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTFP_MAX_MATERIALS 4
#define CTFP_MAX_ENERGIES 256

typedef enum ctfp_status {
    CTFP_OK = 0,
    CTFP_INVALID_ARG = 1,
    CTFP_OOM = 2,
    CTFP_CUDA_ERROR = 3,
    CTFP_TIMEOUT = 4,
    CTFP_UNSUPPORTED = 5,
    CTFP_NOT_READY = 6
} ctfp_status;

/* Scan geometry: the fields of CTScanParas (Source/DataType.h:33-55) that the
 * projector reads, with the reference's names and units (mm, counts). */
typedef struct ctfp_geometry {
    int64_t pNumX, pNumY, pNumZ;        /* phantom voxels                        */
    float pLengthX, pLengthY, pLengthZ; /* phantom size, mm                      */
    int64_t projNum;                    /* views over 360 degrees                */
    int64_t dNumU, dNumV;               /* detector columns, rows                */
    float dSize;                        /* detector pitch, mm                    */
    float sod, sdd;                     /* source-object, source-detector, mm    */
    int32_t rotatedDirection;           /* +1 counter-clockwise, -1 clockwise    */
    int32_t reserved;                   /* must be 0                             */
} ctfp_geometry;

/* Derived quantities: CTScanSystemInfo (Source/DataType.h:78-111) exactly as
 * CBCTForwardProj::computeParas computes them in FP32
 * (Source/CBCTForwardProj.cpp:23-62). */
typedef struct ctfp_system_info {
    float thetaStep, dHalfLU, dHalfLV, FOVR, FOVH;
    float pHalfX, pHalfY, pHalfZ;
    float pSizeX, pSizeY, pSizeZ;
    float dx, dy, dz;
    int64_t intNum; /* samples per ray, K */
} ctfp_system_info;

/* How a material volume is sampled at a ray point. */
typedef enum ctfp_interp {
    /* exact FP32 software trilinear at the reference's sample coordinates */
    CTFP_INTERP_TRILINEAR = 0,
    /* software trilinear with the weights quantised to 8 fractional bits, as
     * the texture unit does for the reference's tex3D (CBCTPolyProjGPU.cu:1920) */
    CTFP_INTERP_TEXEMU = 1,
    /* hardware tex3D on a cudaArray, the reference's own sampler
     * (CBCTPolyProjGPU.cu:2175-2209: border addressing, linear filter) */
    CTFP_INTERP_TEXTURE = 2
} ctfp_interp;

/* Where the software samplers (TRILINEAR, TEXEMU) read a sample's 8 corners. */
typedef enum ctfp_sampler {
    /* the caller's linear volumes through L1 (8 loads per corner set) */
    CTFP_SAMPLER_GLOBAL = 1,
    /* plan-owned layered 2D textures, one layer per z slice: two texture
     * gathers (tld4) return the 8 corners; weights stay in software.  The
     * default where the axis sampler does not fit; needs pNumZ <= 2048. */
    CTFP_SAMPLER_LAYERED = 2,
    /* the caller's linear volumes staged per ray bundle in shared memory: each
     * CTA (8 x 16 rays, one view at a time) copies the voxel box its rays cross
     * in the next 16 samples and reads corners from there.  The copy is one TMA
     * tensor load per material (cp.async.bulk.tensor) when pNumX is a multiple
     * of 4 and every volume starts on a 16-byte boundary, else plain loads;
     * CTFP_BRICK_STAGING=loads forces plain loads. */
    CTFP_SAMPLER_BRICK = 3,
    /* plan-owned layered 2D textures along the two in-plane axes: one copy per
     * material layered along x (a layer per x index, texels (y, z)) and one
     * layered along y.  Each view marches the copy layered along the axis its
     * central ray runs closest to, so consecutive samples of a ray mostly keep
     * their 2x2 in-layer footprint or move it one layer on; the gathers a ray
     * already holds are kept in registers and only the missing layers are
     * fetched.  Results agree with the layered sampler to FP32 rounding (the
     * layer axis is interpolated last).  The default; needs pNumX, pNumY <= 2046
     * and pNumZ <= 32768 (else the layered sampler, else the global one). */
    CTFP_SAMPLER_AXIS = 4
} ctfp_sampler;

/* Grid transmission table layout for ctfp_set_spectral_tables. */
typedef enum ctfp_grid_layout {
    CTFP_GRID_NONE = 0,   /* no anti-scatter grid: G = 1                 */
    CTFP_GRID_COLUMN = 1, /* [E][dNumU], the reference's Grid::updataGrid */
    CTFP_GRID_PIXEL = 2   /* [E][dNumV][dNumU], per-pixel per-energy      */
} ctfp_grid_layout;

typedef struct ctfp_plan ctfp_plan;

/* ---- geometry ------------------------------------------------------------ */

/* CBCTForwardProj::computeParas (Source/CBCTForwardProj.cpp:23-62). */
ctfp_status ctfp_compute_paras(const ctfp_geometry* g, ctfp_system_info* out);

/* View angle in radians, FP32 as the reference's launchers compute it
 * (CBCTPolyProjGPU.cu:51): rotatedDirection * p * thetaStep / 180 * acosf(-1). */
ctfp_status ctfp_view_angle(const ctfp_geometry* g, int64_t view, float* angle);

/* ---- plans ---------------------------------------------------------------- */

/* Replaces initDevice{,SinMat,SinMatNoResponse}{Grid,NoGrid}
 * (CBCTPolyProjGPU.cu:478-1764) without their cudaDeviceReset, without the
 * 3*K*U*V coordinate buffers and without the K*U*V sample buffer. */
ctfp_status ctfp_plan_create(const ctfp_geometry* g, int32_t n_materials, int32_t interp,
                             int32_t device, ctfp_plan** out);
/* Replaces freeDeviceMemory (CBCTPolyProjGPU.cu:1774-1797). */
ctfp_status ctfp_plan_destroy(ctfp_plan* plan);
ctfp_status ctfp_plan_get_system_info(const ctfp_plan* plan, ctfp_system_info* out);
ctfp_status ctfp_plan_set_interp(ctfp_plan* plan, int32_t interp);
ctfp_status ctfp_plan_set_sampler(ctfp_plan* plan, int32_t sampler);
/* Ray-tile shape of the march kernels: tile_u x tile_v pixels per CTA (a
 * multiple of 32 threads, at most 256), views_per_cta views marched by each
 * CTA for its tile, and min_ctas_per_sm (2, 3, 4, or 5 for the axis sampler;
 * other samplers run 5 as 4), the residency the forward march is compiled for
 * (its register cap: 65536 / (256 * min_ctas_per_sm)).
 * Set by the autotuner; defaults 16 x 8 x 2 x 4. */
ctfp_status ctfp_plan_set_launch_shape(ctfp_plan* plan, int32_t tile_u, int32_t tile_v, int32_t views_per_cta,
                                       int32_t min_ctas_per_sm);

/* Empty-space skipping (off by default) for the layered sampler
 * (CTFP_INTERP_TRILINEAR, CTFP_INTERP_TEXEMU) and the hardware texture
 * (CTFP_INTERP_TEXTURE).  Each call first marks the 8^3-voxel bricks (dilated
 * by one voxel) that hold a non-zero voxel of any material; the march then
 * skips samples whose 2x2x2 footprint lies in an unmarked brick, whose
 * contribution is exactly zero.  Results equal the full march up to FP32
 * rounding of the compensated sums.  The global and brick samplers march every
 * sample.  No counterpart in the reference. */
ctfp_status ctfp_plan_set_skip_empty(ctfp_plan* plan, int32_t enable);

/* Bits of the plan's status word (ctfp_plan_check_status). */
#define CTFP_STATUS_WAIT_TIMEOUT 1u      /* a staging wait ran out; outputs still correct */
#define CTFP_STATUS_EXIT_WAIT_TIMEOUT 2u /* the wait at CTA exit ran out too; outputs not trusted */

/* Waits for the device, then reads and clears the plan's status word: flags
 * receives its bits (may be NULL).  Returns CTFP_TIMEOUT when a kernel of the
 * plan gave up a bounded wait since the last check: a CTA of the TMA-staged
 * brick sampler whose tensor load did not complete within CTFP_WAIT_LIMIT
 * polls (default 65536) read those samples from the volume instead and stopped
 * staging, so its outputs are still correct (CTFP_STATUS_WAIT_TIMEOUT).
 * Returns CTFP_CUDA_ERROR when such a CTA's second bounded wait, before it
 * exits, also ran out (CTFP_STATUS_EXIT_WAIT_TIMEOUT): the abandoned copy may
 * have landed in shared memory that another CTA then owned, so the plan's
 * outputs since the last check are not to be trusted.  No counterpart in the
 * reference, whose launchers printed CUDA errors and carried on
 * (Source/CUDAFun/CBCTPolyProjGPU.cu:55-61). */
ctfp_status ctfp_plan_check_status(ctfp_plan* plan, uint32_t* flags);

/* Focal spot (CBCTSinMatPolyForwardProj{Grid,NoGrid}::computePolyForwProjFoSp,
 * Source/CBCTSinMatPolyForwardProjGrid.cpp:269-388, CBCTPolyProjGPU.cu:1927-1978):
 * per-view source offsets offset_u, offset_v [projNum] in mm (host arrays,
 * copied; both NULL clears).  The forward then samples each view with its
 * offset added to the rotated y and the z coordinate, re-aligns the view's
 * line-integral images by (offset_u, offset_v) / dSize detector pixels with
 * bilinear interpolation (texture-unit weights in the compat modes, exact in
 * CTFP_INTERP_TRILINEAR; 0 outside the image), and runs the spectral epilogue
 * on the re-aligned integrals; an L checkpoint holds the re-aligned integrals.
 * The reference's path exists for single-material phantoms; here every
 * material is re-aligned alike.  The adjoint (ctfp_backward*) and the batched
 * form return CTFP_UNSUPPORTED while a focal spot is set. */
ctfp_status ctfp_plan_set_focal_spot(ctfp_plan* plan, const float* offset_u, const float* offset_v);
/* The reference's offsets: srand(10), MSVC rand(), a 1e-4 mm lattice over
 * [-size/2, size/2), redrawn while u^2 + v^2 > pi * (size/2)^2
 * (CBCTForwardProj::computeFoSpOffset, Source/CBCTForwardProj.cpp:122-148). */
ctfp_status ctfp_focal_spot_offsets(int64_t n_views, float focal_spot_size, float* offset_u, float* offset_v);

/* Spectral tables, host pointers, copied into the plan.
 *   spectrum     [E]     normalised spectrum S_e
 *   mu           [E][M]  per-material attenuation per unit density, 1/mm per
 *                        g/cm^3, i.e. (mu/rho)(E)/10 (PhantomObject.cpp:56,62)
 *   grid         NULL or [E][dNumU] / [E][dNumV][dNumU] per grid_layout
 *   det_response NULL (D = 1) or [E][dNumV][dNumU]
 *                (CBCTForwardProj.cpp:114-120 per energy)
 *   I0Val        photons per pixel before weighting (CTScanParas::I0Val)
 * Builds the per-pixel energy weights W_e = I0Val*S_e*G_e*D_e and the flat
 * field I0 = sum_e W_e (CBCTPolyForwardProjGrid.cpp:330-350). */
ctfp_status ctfp_set_spectral_tables(ctfp_plan* plan, int32_t n_energies, const float* spectrum,
                                     const float* mu, const float* grid, int32_t grid_layout,
                                     const float* det_response, float I0Val);

/* ---- forward -------------------------------------------------------------- */

/* Per-ray material path integrals L_m = dx * sum_i interp(rho_m, x_i)
 * (transformKernel + computeSinMatIndensityProjKernel, CBCTPolyProjGPU.cu:1902-1924,
 * 2005-2020), written to L [projNum][dNumV][dNumU][M]. volumes: M device
 * pointers (host array). */
ctfp_status ctfp_line_integrals(ctfp_plan* plan, const float* const* volumes, float* L, void* stream);

/* Fused ray march + spectral epilogue. Replaces the per-energy, per-view loop
 * of forward{,SinMat,SinMatNoResponse}Proj{Grid,NoGrid}GPU (CBCTPolyProjGPU.cu:12-474)
 * and the host sum over energies (CBCTForwardProj.cpp:65-76):
 *   I   = sum_e W_e exp(-sum_m mu[e][m] L_m)
 *   IAbs= sum_e W_e (1 - exp(-sum_m mu[e][m] L_m))
 * I, IAbsorb: device [projNum][dNumV][dNumU]; I0 (device [dNumV][dNumU]) and
 * L_ckpt (device [projNum][dNumV][dNumU][M]) may be NULL. */
ctfp_status ctfp_forward(ctfp_plan* plan, const float* const* volumes, float* I, float* IAbsorb,
                         float* I0, float* L_ckpt, void* stream);

/* ctfp_forward with HOST buffers, the shape of the reference's per-energy
 * launchers (CBCTPolyProjGPU.cu:12-109: host volume in, host I/IAbsorb out):
 * copies the M host volumes to plan-owned device buffers, runs the forward in
 * up to 16 chunks of views and copies each chunk's I, IAbsorb (host
 * [projNum][dNumV][dNumU]) back on a plan-owned stream while the next chunk is
 * marched, then I0 (host [dNumV][dNumU], may be NULL), and synchronises the
 * stream.  The chunks alternate between the given stream and a second
 * plan-owned stream, so one chunk's last wave overlaps the next chunk's first
 * (with a focal spot set they all run on the given stream).  Page-locked host
 * buffers make the copies asynchronous DMA (and let them overlap the march). */
ctfp_status ctfp_forward_host(ctfp_plan* plan, const float* const* host_volumes, float* host_I,
                              float* host_IAbsorb, float* host_I0, void* stream);

/* Spectral epilogue alone from given path integrals L (e.g. the single-material
 * path's density projection, forwardSin*Kernel, CBCTPolyProjGPU.cu:2046-2169). */
ctfp_status ctfp_spectral_from_L(ctfp_plan* plan, const float* L, float* I, float* IAbsorb, void* stream);

/* Compat outputs (CBCTForwardProj.cpp:79-90, 376-387): Ipoly = floor(I) as
 * uint32, IAbsPoly = floor(IAbsorb), proj = logf(I0 / Ipoly). n_pix = U*V.
 * Any output pointer may be NULL. */
ctfp_status ctfp_finalize_counts(int64_t n_pix, int64_t n_views, const float* I, const float* IAbsorb,
                                 const float* I0, uint32_t* Ipoly, uint32_t* IAbsPoly, float* proj,
                                 void* stream);

/* ---- adjoint (no reference counterpart) ------------------------------------ */

/* Gradient of a loss with respect to each material density map, given dLoss/dI
 * (gI) and optionally dLoss/dIAbsorb (gIAbsorb, may be NULL), both
 * [projNum][dNumV][dNumU], and the L checkpoint written by ctfp_forward.
 * Accumulates (+=) into g_volumes (M device pointers, same layout as volumes):
 *   gL_m   = (gIAbs - gI) * sum_e mu[e][m] W_e exp(-sum_k mu[e][k] L_k)
 *   g_rho_m[x] += dx * sum_{rays, i} w_i(x) gL_m     (transposed trilinear weights)
 * In CTFP_INTERP_TEXTURE mode the transposed weights are the quantised
 * texture weights (CTFP_INTERP_TEXEMU). */
ctfp_status ctfp_backward(ctfp_plan* plan, const float* L_ckpt, const float* gI, const float* gIAbsorb,
                          float* const* g_volumes, void* stream);

/* Transpose of ctfp_line_integrals: g_volumes[m][x] += dx * sum w_i(x) gL[ray][m]. */
ctfp_status ctfp_line_integrals_adjoint(ctfp_plan* plan, const float* gL, float* const* g_volumes,
                                        void* stream);

/* ---- sampler roofline --------------------------------------------------------
 * No counterpart in the reference.  Measures, on `device`, the peak rate at
 * which the texture path delivers trilinear footprints with nothing else to
 * do: kind CTFP_SAMPLER_LAYERED times two 4-texel gathers (tld4) per
 * voxel-sample, kind 0 one filtered tex3D fetch (the CTFP_INTERP_TEXTURE
 * path), both from a texture that stays in the L1 texture cache, at full
 * occupancy, with the march's warp shape.  Writes voxel-samples per second. */
ctfp_status ctfp_sampler_peak(int32_t device, int32_t kind, double* voxel_samples_per_s);

/* No counterpart in the reference.  The texture-emulation mode's sample
 * coordinates divide by the voxel size as the reference does, with the
 * quotient formed from the plan's FP32 reciprocal of the divisor and two
 * exact-remainder correction steps instead of an IEEE division.  This check runs that
 * arithmetic on n pseudo-random dividends (both signs, magnitudes 2^-20 to
 * 2^21, seeded) against the device's IEEE division by `divisor` and writes the
 * number of results that differ in any bit (0 expected). */
ctfp_status ctfp_check_division(int32_t device, float divisor, int64_t n, uint64_t seed, int64_t* mismatches);

/* ---- launch-shape autotuner ------------------------------------------------
 * No counterpart in the reference (fixed 8 x 8 x 8 blocks,
 * Source/CUDAFun/CBCTPolyProjGPU.cuh:22-24).  Times candidate launch shapes of
 * the fused forward (tiles 8 x 8 ... 64 x 4, 2-4 CTAs per SM, 1-4 views per CTA)
 * on n_sample_views views (0: 64) in four chunks spread round the rotation,
 * run concurrently, and sets the fastest on the plan (as
 * ctfp_plan_set_launch_shape).  The sample ends in a partial wave of CTAs that
 * weighs more for CTAs of more views, so short samples lean towards 1 view per
 * CTA: on the 256^3 two-material 360-view workload 64 sample views pick what
 * all 360 pick (2 views per CTA), 16 pick 1 view per CTA, 5 % slower on the
 * whole forward.  Tuning takes about 36 forwards of the sample.  I and IAbsorb
 * are full-size output buffers as for ctfp_forward; their contents are
 * undefined afterwards.  Synchronises the stream.  Results are cached per
 * process by geometry, materials, sampler, energies and device name, and in the
 * text file named by the environment variable CTFP_TUNE_CACHE when it is set. */
typedef struct ctfp_launch_shape {
    int32_t tile_u, tile_v, views_per_cta, min_ctas_per_sm;
    float ms;            /* time of the sampled views with this shape */
    int32_t from_cache;  /* 1 when no timing ran */
} ctfp_launch_shape;
ctfp_status ctfp_plan_autotune(ctfp_plan* plan, const float* const* volumes, float* I, float* IAbsorb,
                               int32_t n_sample_views, ctfp_launch_shape* out, void* stream);

/* ---- batched form -------------------------------------------------------------
 * No counterpart in the reference, which simulates one phantom per process run
 * (Source/Main_Forward_Projection_V1.1.cpp:18-23).  A batch holds n_items plans (own geometry, materials,
 * spectral tables; one device) and runs them with persistent kernels over a
 * device work queue: a forward work unit is one view x one 8 x 16 detector
 * tile (the 128 rays of one CTA), a fused forward + adjoint unit one view x
 * one 8 x 8 tile (64 rays; see ctfp_batch_set_shape, ctfp_batch_set_views
 * and ctfp_batch_autotune for other shapes); items are grouped by material count and sampler mode
 * (one kernel per group, each with its own register budget) and queued
 * largest first (rays x samples x materials); every CTA takes the next unit
 * from an atomic counter.  A call is recorded once as a CUDA graph (volume
 * uploads, queue reset, kernels, fold) and replayed, in the order of the
 * stream passed, while the item pointers and the plans' tables stay the same;
 * a change re-records it (one host synchronisation).  The batch uploads into
 * the plans' own texture arrays: do not run a batch and its plans
 * concurrently.
 *
 * Items use the axis sampler (the default) or the layered one in
 * CTFP_INTERP_TRILINEAR or CTFP_INTERP_TEXEMU, or CTFP_INTERP_TEXTURE
 * (hardware tex3D; its adjoint is the
 * transpose of the texture unit's weights, as ctfp_backward), have no focal
 * spot and have spectral tables set.  The batch keeps the
 * plans' pointers: destroy it before them.  Arrays indexed by item follow the
 * order of `plans`. */
typedef struct ctfp_batch ctfp_batch;
ctfp_status ctfp_batch_create(int32_t n_items, ctfp_plan* const* plans, ctfp_batch** out);
ctfp_status ctfp_batch_destroy(ctfp_batch* batch);

/* Per item k: the same outputs as ctfp_forward(plans[k], volumes[k], I[k],
 * IAbsorb[k], NULL, L_ckpt[k]).  IAbsorb and L_ckpt may be NULL (whole array)
 * or hold NULL entries. */
ctfp_status ctfp_batch_forward(ctfp_batch* batch, const float* const* const* volumes, float* const* I,
                               float* const* IAbsorb, float* const* L_ckpt, void* stream);

/* Fused forward + loss + adjoint.  Per item k and ray r, with I_r the forward
 * intensity and T_r = I_target[k][r] > 0:
 *   loss[k]         = sum_r (log I_r - log T_r)^2            (device, may be NULL)
 *   g_volumes[k][m] += d loss[k] / d volumes[k][m]           (accumulated)
 * rays with I_r <= 0 contribute nothing.  I (may be NULL) receives I_r. */
ctfp_status ctfp_batch_forward_adjoint(ctfp_batch* batch, const float* const* const* volumes,
                                       const float* const* I_target, float* const* I,
                                       float* const* const* g_volumes, float* loss, void* stream);

/* Work units in the queue, persistent grid sizes of the two kernels. */
/* Ray tile of a fused forward + adjoint work unit (one view): tile_u x tile_v
 * rays, whose product must be 64, the threads of its persistent CTA, with
 * tile_u a power of two (default 8 x 8); the forward's units get the same
 * tile twice as high (tile_u x 2 tile_v, 128 threads, two views).  Waits for
 * the device; the next call re-records its graph. */
ctfp_status ctfp_batch_set_shape(ctfp_batch* batch, int32_t tile_u, int32_t tile_v);
/* Views of a work unit, per kind of call (1 to 8, default 1): a unit marches
 * its rays for that many consecutive views, one after the other, so the
 * unit's queue atomic, barriers and item lookup are spread over more rays.
 * Waits for the device; the next call re-records its graph. */
ctfp_status ctfp_batch_set_views(ctfp_batch* batch, int32_t fwd_views, int32_t adj_views);
ctfp_status ctfp_batch_get_views(const ctfp_batch* batch, int32_t* fwd_views, int32_t* adj_views);
/* Times, for each kind of call on its own, the forward and the fused forward
 * + loss + adjoint kernels on the first eighth of every group's work queue
 * (its largest problems): the candidate ray tiles (8 x 8, 16 x 4, 4 x 16,
 * 32 x 2, 2 x 32; the forward's twice as high) at the kind's current views
 * per unit, then 1, 2 and 4 views per unit with the fastest tile, and keeps
 * the fastest tile and views of each kind.  Reads volumes and I_target as
 * ctfp_batch_forward_adjoint does and writes nothing the caller owns; out
 * (may be NULL) receives the fused kernel's tile_u, tile_v, views_per_cta and
 * ms (ctfp_batch_get_shapes and ctfp_batch_get_views return both kinds').
 * Waits for the device. */
ctfp_status ctfp_batch_autotune(ctfp_batch* batch, const float* const* const* volumes, const float* const* I_target,
                                ctfp_launch_shape* out, void* stream);
ctfp_status ctfp_batch_info(const ctfp_batch* batch, int64_t* total_units, int32_t* grid_forward,
                            int32_t* grid_adjoint);
/* The work-unit ray tiles of the forward and of the fused forward + adjoint
 * calls (any pointer may be NULL). */
ctfp_status ctfp_batch_get_shapes(const ctfp_batch* batch, int32_t* fwd_tile_u, int32_t* fwd_tile_v,
                                  int32_t* adj_tile_u, int32_t* adj_tile_v);

/* ---- view ranges (sharding one object's views across GPUs) -----------------
 * No counterpart in the reference.  The forward and the adjoint over views
 * [view0, view0 + n_views) only, with compact buffers: I, IAbsorb, L_ckpt,
 * gI and gIAbsorb hold those views from index 0 ([n_views][dNumV][dNumU],
 * L_ckpt [n_views][dNumV][dNumU][M]).  Each GPU of a view-sharded projection
 * runs its own range on its own plan; the gradient volumes are partial sums
 * over the range (sum them across GPUs).  n_views = 0 is a no-op. */
ctfp_status ctfp_forward_views(ctfp_plan* plan, const float* const* volumes, int64_t view0, int64_t n_views,
                               float* I, float* IAbsorb, float* I0, float* L_ckpt, void* stream);
ctfp_status ctfp_backward_views(ctfp_plan* plan, const float* L_ckpt, const float* gI, const float* gIAbsorb,
                                int64_t view0, int64_t n_views, float* const* g_volumes, void* stream);

/* ---- forward without device allocation -------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code running inside a host framework that owns all device memory through its
 * own pool, real-time loops that must not allocate after start-up, or processes
 * held to a fixed memory budget on a shared GPU.  ctfp_forward needs a plan, and
 * a plan allocates its tables; this entry point allocates nothing.
 *
 * It runs the same fused march + spectral epilogue as ctfp_forward on the
 * calling thread's current device.  The caller passes every input and output:
 * spectrum [E] and mu [E][M] (host), grid (device: NULL, [E][dNumU] or
 * [E][dNumV][dNumU] per grid_layout), det_response (device, NULL or
 * [E][dNumV][dNumU]), volumes (M device pointers), I and IAbsorb (device
 * [projNum][dNumV][dNumU]) and I0 (device [dNumV][dNumU], may be NULL).  The
 * energy weights I0Val*S*G*D are formed per ray instead of being tabulated.
 *
 * Its scratch (per-view trigonometry, the attenuation and spectrum tables) is a
 * fixed array of CTFP_NOALLOC_SCRATCH_BYTES in the library's device module,
 * which every GPU that loads the library holds until the process exits.  Limits:
 * projNum <= CTFP_NOALLOC_MAX_VIEWS, n_energies <= CTFP_MAX_ENERGIES,
 * n_materials <= CTFP_MAX_MATERIALS; larger sizes return CTFP_INVALID_ARG.
 * interp must be CTFP_INTERP_TRILINEAR or CTFP_INTERP_TEXEMU (the hardware
 * texture needs a cudaArray).  Every call copies its host tables (spectrum,
 * mu, the views' trigonometry) from pageable host memory, which a CUDA graph
 * capture cannot record: a call on a stream that is capturing returns
 * CTFP_UNSUPPORTED and issues nothing.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress).  That address is cached per
 * device index for the life of the
 * process: after the caller resets a device (cudaDeviceReset) the cached address
 * no longer names the array, so a process that resets a device must not call
 * this entry point on it again.  All calls on a device share the array and it
 * keeps the last call's contents: calls whose work overlaps on the GPU
 * (different streams or threads) race on it and must be serialised by the
 * caller.  Speed: it reads each sample's 8 corners with plain loads from the
 * caller's volumes (no plan-owned texture copies), about 3.6x the time of
 * ctfp_forward's texture gathers on the 256^3 two-material grid workload. */
#define CTFP_NOALLOC_MAX_VIEWS 8192
#define CTFP_NOALLOC_SCRATCH_BYTES (200 * 1024)
ctfp_status ctfp_forward_noalloc(const ctfp_geometry* g, int32_t n_materials, int32_t interp, int32_t n_energies,
                                 const float* spectrum, const float* mu, const float* grid, int32_t grid_layout,
                                 const float* det_response, float I0Val, const float* const* volumes, float* I,
                                 float* IAbsorb, float* I0, void* stream);

/* ---- table builders on the device -------------------------------------- */

/* Focused anti-scatter grid geometry, GridInfo (Source/DataType.h:57-75). */
typedef struct ctfp_grid_params {
    int32_t gridStripsWidth;  /* um, integer (Grid.h:6-8)  */
    int32_t interspaceWidth;  /* um, integer               */
    float h;                  /* grid height, mm           */
    float FD;                 /* focal distance, mm        */
} ctfp_grid_params;

/* Grid transmission per energy, written to device memory `out`:
 *   layout CTFP_GRID_COLUMN: [E][dNumU], the reference's 1-um discretised
 *     focused strip grid averaged over each detector column
 *     (Grid::defGrid/updataGrid/binning1D, Grid.cpp:76-309, 373-443), including
 *     its quirk that an interspace takes the period-start unit's height
 *     (Grid.cpp:115);
 *   layout CTFP_GRID_PIXEL: [E][dNumV][dNumU], the same strip pattern with the
 *     slant path through the grid taken from the full incidence angle of the ray
 *     to each pixel, h * sqrt(FD^2 + d_u^2 + d_v^2) / FD (reduces to the column
 *     table on the central row).
 * mu_strip, mu_inter: host [E], linear attenuation in 1/mm (the mass tables
 * times density / 10, CBCTForwardProj.cpp:196, 220).  dSize*1000 must be an
 * integer number of um. */
ctfp_status ctfp_build_grid_table(const ctfp_geometry* g, const ctfp_grid_params* grid, int32_t n_energies,
                                  const float* mu_strip, const float* mu_inter, int32_t layout, float* out,
                                  void* stream);

/* Per-pixel scintillator thickness with the reference's seeded jitter
 * (CBCTForwardProj::computePerScinThinckness, CBCTForwardProj.cpp:99-111):
 * srand(100) and the MSVC CRT rand() the reference was built with.  Host
 * output [n_pix]. */
ctfp_status ctfp_scintillator_thickness(int64_t n_pix, float thickness, float thickness_err, float* out);

/* Detector response per energy on the device (CBCTForwardProj::updateDetResponse,
 * CBCTForwardProj.cpp:114-120): out[e][k] = factor * (1 - exp(-mu_scint[e] * t[k])).
 * mu_scint: host [E] in 1/mm; thickness: device [n_pix]; out: device [E][n_pix]. */
ctfp_status ctfp_build_det_response(int32_t n_energies, int64_t n_pix, const float* mu_scint,
                                    const float* thickness, float factor, float* out, void* stream);

/* Label map -> M density maps on the device (PhantomObject::updataLineAtten /
 * computeDesity, PhantomObject.cpp:38-71): out[m][x] = density[m] if
 * labels[x] == m + 1 else 0.  labels: device uint8 [n_vox]; density: host [M];
 * out: M device pointers. */
ctfp_status ctfp_labels_to_density(const uint8_t* labels, int64_t n_vox, int32_t n_materials,
                                   const float* density, float* const* out, void* stream);

/* ---- diagnostics ----------------------------------------------------------- */

/* Samples one volume [nz][ny][nx] at n points (device float3 array of
 * continuous voxel coordinates, voxel i at i) with the given interp mode,
 * border 0. Used to pin the texture emulation against the hardware sampler. */
ctfp_status ctfp_sample_volume(const float* volume, int64_t nx, int64_t ny, int64_t nz, int32_t interp,
                               const float* points, int64_t n, float* out, void* stream);

/* Exact number of (ray, sample) pairs whose trilinear footprint touches the
 * volume, i.e. the samples the march evaluates (others contribute exactly 0). */
ctfp_status ctfp_count_support_samples(ctfp_plan* plan, int64_t* out);

/* The texture work of the axis sampler's march on this plan's geometry with
 * its launch shape: every view's rays are stepped as the march steps them
 * and, per iteration of a warp and per gather slot, the 4-lane quads with a
 * lane that fetches are counted (the texture unit spends its time per active
 * quad).  quad_gathers_per_sample = quads counted / (ray, sample) pairs
 * evaluated, per material.  Fetching both slots on every sample in full warps
 * (as the layered sampler's two gathers do) gives 0.5 (16 quads per 32
 * samples), so the axis march's texture roof is ctfp_sampler_peak
 * (CTFP_SAMPLER_LAYERED) x 0.5 / quad_gathers_per_sample voxel-samples/s.
 * Does not depend on the volumes.  No counterpart in the reference. */
ctfp_status ctfp_axis_gather_count(ctfp_plan* plan, double* quad_gathers_per_sample);

/* Message of the last error on the calling thread ("" if none). */
const char* ctfp_last_error_string(void);

/* Library version string. */
const char* ctfp_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CTFP_H */
