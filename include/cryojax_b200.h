/*
 * cryojax_b200 — C-ABI of the B200 (sm_100a) Fourier-slice + CTF image path.
 *
 * Plain C: pointers, sizes and POD structs only.  Every device pointer is a
 * CUDA global-memory address on the current device; `stream` is a
 * cudaStream_t passed as void*.  All work is stream-ordered: no entry point
 * synchronises the device or allocates device memory unless it says so.
 * Every entry point returns CJX_OK (0) or a nonzero CJX_ERR_* code;
 * cjx_get_last_error() returns the calling thread's last message.
 *
 * Data conventions follow cryoJAX exactly:
 *   - volume grid: the full, centred (fftshifted) 3-D FFT of the padded real
 *     volume, complex64, C-order [z][y][x], side N
 *     (FourierVoxelGridVolume.fourier_voxel_grid,
 *      cryojax/simulator/_volume/representations/voxel_volume.py:40-119);
 *   - image output: rfft half-plane, complex64, C-order [Py][Px/2+1], zero
 *     frequency in the corner (cryojax/ndimage/_fft.py:80-99 conventions).
 */
#ifndef CRYOJAX_B200_H
#define CRYOJAX_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CJX_API __attribute__((visibility("default")))
#else
#define CJX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CJX_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------- */
/* Device arrays: complex64 grids, images and outputs must be 8-byte
 * aligned, x-pair grids (CJX_GRID_BRICKED_PAIRS) 16-byte aligned; the
 * entry points return CJX_ERR_INVALID_ARGUMENT otherwise.                 */
#define CJX_OK 0
#define CJX_ERR_INVALID_ARGUMENT 1 /* bad shape, null pointer, bad flag,
                                      misaligned array                    */
#define CJX_ERR_UNSUPPORTED 2      /* size beyond the compiled limits     */
#define CJX_ERR_CUDA 3             /* a CUDA runtime call failed          */
#define CJX_ERR_WORKSPACE 4        /* workspace too small                  */

/* ---- limits ------------------------------------------------------------ */
#define CJX_MAX_SIDE 1024 /* max volume side N and max image side Py, Px */

/* ---- flags for cjx_slice_desc.flags ----------------------------------- */
/* multiply by the AstigmaticCTF of ContrastTransferTheory
 * (cryojax/simulator/_transfer_theory/transfer_theory.py:53-119)          */
#define CJX_APPLY_CTF (1u << 0)
/* zero the even-size Nyquist self-conjugates, then multiply by
 * exp(-2 pi i q.t) (cryojax/simulator/_pose.py:68-114)                    */
#define CJX_APPLY_TRANSLATION (1u << 1)
/* multiply by envelope_amplitude * exp(-b/4 k^2) (FourierGaussian,
 * cryojax/ndimage/operators/_fourier_operator.py:183-234)                 */
#define CJX_APPLY_ENVELOPE (1u << 2)
/* out-of-bounds corners with a negative index read the fill value instead
 * of wrapping to index + N.  NOT the reference's behaviour (JAX's
 * `.at[].get(mode="fill")` wraps negative indices once); offered for
 * comparison only.                                                        */
#define CJX_ZERO_FILL_NEGATIVE (1u << 3)
/* `grid` is in the bricked layout written by cjx_brick_volume instead of
 * the reference's C-order array.                                          */
#define CJX_GRID_BRICKED (1u << 4)
/* `grid` is in the x-pair layout written by cjx_brick_volume_pairs: the
 * bricked order with 16-byte entries (g(x), g(x+1)), so that an interior
 * trilinear sample reads its 8 corners with 4 vector loads.  Forward,
 * search and (voxel grids) loss-gradient entry points.                    */
#define CJX_GRID_BRICKED_PAIRS (1u << 5)
/* `grid` holds the cubic-spline coefficients of a FourierVoxelSplineVolume
 * (side N + 2: C order, bricked on side N + 2 with CJX_GRID_BRICKED,
 * or x-pair bricked on side N + 2 with CJX_GRID_BRICKED_PAIRS, as written
 * by cjx_brick_volume / cjx_brick_volume_pairs with n = N + 2)
 * instead of the voxel grid, and every sample is the reference's 4x4x4-tap
 * cubic-spline interpolation
 * (cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:148-183,
 * 453-462, 531-534; cryojax/ndimage/_map_coordinates.py:126-142, 217-250).
 * desc->n stays the voxel grid's side N.  Forward, multi, no-alloc and
 * search entry points, and cjx_slice_ctf_loss_grad (C order or bricked;
 * grid_grad is then the (N + 2)^3 C-order coefficient gradient).           */
#define CJX_GRID_SPLINE (1u << 6)
/* EwaldSphereExtraction instead of FourierSliceExtraction
 * (cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:225-516):
 * the full N x N surface at R (kx, ky, lambda (kx^2 + ky^2) / (2 N
 * pixel_size)) (pixel frequency indices) is sampled, with no rfft-half
 * conversion, and resized with complex FFTs.  With CJX_APPLY_CTF the output
 * is ContrastTransferTheory's non-projection contrast
 * (cryojax/simulator/_transfer_theory/transfer_theory.py:100-111, 165-255),
 * [Py][Px/2+1], from amplitude_contrast_ratio and phase_shift of the
 * parameter record; CJX_APPLY_ENVELOPE and CJX_APPLY_TRANSLATION as usual.
 * Without CJX_APPLY_CTF the output is the integrator's full spectrum
 * [Py][Px] (scale applied; no envelope or translation allowed).  Any grid
 * layout, trilinear or spline.  Forward, multi and no-alloc entry points,
 * cjx_search with CJX_APPLY_CTF (the scores are the contrast images'
 * NCC) and cjx_slice_ctf_loss_grad with CJX_APPLY_CTF.                    */
#define CJX_EWALD_SPHERE (1u << 7)

/* ---- per-image parameters (one record per image, device memory) ------
 * 32 doubles (256 bytes).  Built on the host from a pose, a CTF and an
 * image config.                                                            */
typedef struct cjx_image_params {
  double rot[9];              /* row-major R; sample point = R (kx, ky, 0)
                                 (QuaternionPose.rotation applied with
                                 SO3.apply, cryojax/simulator/_pose.py:29-66) */
  double shift_x, shift_y;    /* in-plane offset, Angstrom                  */
  double defocus;             /* mean defocus + out-of-plane offset, A      */
  double astigmatism;         /* Angstrom                                   */
  double astigmatism_angle;   /* radians                                    */
  double spherical_aberration;/* Angstrom (mm * 1e7)                        */
  double wavelength;          /* Angstrom                                   */
  double phase_total;         /* radians: deg2rad(phase_shift)
                                 + atan(ac / sqrt(1 - ac^2))                 */
  double pixel_size;          /* Angstrom                                   */
  double scale;               /* prefactor: pixel_size if outputs_integral,
                                 times the interaction constant for the
                                 contrast model, else 1                      */
  double envelope_amplitude;  /* used with CJX_APPLY_ENVELOPE               */
  double envelope_b_factor;   /* Angstrom^2                                 */
  double amplitude_contrast_ratio; /* CJX_EWALD_SPHERE with CJX_APPLY_CTF  */
  double phase_shift;         /* radians: deg2rad(phase_shift), same use    */
  double reserved[9];
} cjx_image_params;

/* ---- geometry of one launch ------------------------------------------- */
typedef struct cjx_slice_desc {
  int32_t n;                 /* volume side N (grid is N^3)                 */
  int32_t py, px;            /* image padded shape (Py, Px)                 */
  uint32_t flags;            /* CJX_* flags above                           */
  float fill_re, fill_im;    /* FourierSliceExtraction.fill_value           */
  int32_t images_per_chunk;  /* resize path: images per workspace chunk;
                                0 = library default                         */
  int32_t reserved;
} cjx_slice_desc;

/* Library ABI version (CJX_ABI_VERSION). */
CJX_API int cjx_get_version(void);

/* Last error message of the calling thread ("" if none). */
CJX_API const char* cjx_get_last_error(void);

/* Workspace needed by cjx_slice_ctf_forward for `n_images` images.
 * Zero when (Py, Px) == (N, N) (no resize stage).  The workspace is
 * scratch: its contents on entry are ignored.                              */
CJX_API int cjx_slice_ctf_workspace_size(const cjx_slice_desc* desc, int64_t n_images,
                                 size_t* bytes);

/* Batched Fourier-slice extraction (+ CTF, envelope, translation).
 *
 * For image b: rotate the central slice by params[b].rot, sample `grid`
 * trilinearly with cryoJAX's out-of-bounds rule, keep the rfft half-plane,
 * resize to (Py, Px) when (Py, Px) != (N, N) (irfftn -> centre crop or pad
 * -> rfftn), multiply by params[b].scale, then apply the flagged CTF,
 * envelope and translation.  Writes out[b][Py][Px/2+1] (complex64).
 *
 * Replaces, for a FourierVoxelGridVolume under eqx.filter_vmap:
 *   flags = CTF|TRANSLATION : LinearImageModel.compute_fourier_image
 *        (cryojax/simulator/_image_model/base_image_model.py:297-328)
 *   flags = 0               : volume.rotate_to_pose(pose) then
 *        FourierSliceExtraction.integrate(..., outputs_real_space=False)
 *        (cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:78-146)
 *   flags = TRANSLATION     : ProjectionImageModel.compute_fourier_image
 *        (cryojax/simulator/_image_model/base_image_model.py:412-432)
 *
 * grid:    device, complex64 [N][N][N]
 * params:  device, n_images records
 * order:   device int32 [n_images], a permutation giving the processing
 *          order (image order[k] is processed k-th; its output still lands
 *          in out[order[k]]), or NULL for 0, 1, 2, ...  Processing images
 *          with similar plane orientations together lets their gathers share
 *          L2 (see cryojax_b200.simulator.orientation_order).
 * out:     device, complex64 [n_images][Py][Px/2+1]
 * workspace: device scratch of at least cjx_slice_ctf_workspace_size bytes
 *          (may be NULL when that size is 0)                              */
CJX_API int cjx_slice_ctf_forward(const cjx_slice_desc* desc, const void* grid,
                                  const cjx_image_params* params, const int32_t* order,
                                  int64_t n_images, void* out, void* workspace,
                                  size_t workspace_bytes, void* stream);

/* ---- squared-residual loss and gradients (reverse mode) -------------- */
/* Per-image result record (16 doubles, device memory).                    */
typedef struct cjx_image_grads {
  double loss;        /* sum over pixels of (x - obs)^2                      */
  double d_shift_x;   /* dL / d shift_x   (Angstrom^-1)                      */
  double d_shift_y;
  double d_defocus;   /* dL / d defocus (the mean defocus incl. offset_z)    */
  double d_rot[6];    /* dL / dR[i][j] for j = 0, 1 (the columns that span
                         the slice plane), row-major [3][2]; chain to the
                         pose parameters on the host                         */
  double d_rot_z[3];  /* dL / dR[i][2] (CJX_EWALD_SPHERE: the surface's third
                         coordinate); zero for the slice                     */
  double reserved[3];
} cjx_image_grads;

/* cjx_slice_ctf_forward with a Fourier-space filter fused into the output
 * epilogue: every output entry [y][x] is multiplied by filter[y][x]
 * (float32, device; the output's own layout: [Py][Px/2+1], or [Py][Px]
 * for the Ewald sphere's full spectrum).  This is
 * AbstractImageModel.postprocess's `filter` applied to the Fourier image
 * (cryojax/simulator/_image_model/base_image_model.py:107-158) before the
 * inverse transform, e.g. cryojax.ndimage's LowpassFilter / HighpassFilter
 * / CustomFilter arrays.  filter = NULL is cjx_slice_ctf_forward.         */
CJX_API int cjx_slice_ctf_forward_filtered(const cjx_slice_desc* desc, const void* grid,
                                           const cjx_image_params* params, const int32_t* order,
                                           int64_t n_images, const float* filter, void* out,
                                           void* workspace, size_t workspace_bytes, void* stream);

/* Workspace for cjx_slice_ctf_loss_grad: the forward's resize-path scratch
 * per chunk of images, then (voxel grids) a bricked N^3 complex64
 * accumulator into which the grid scatter adds before the result goes into
 * grid_grad (its atomics then touch fewer cache lines).  A workspace of only
 * the first part is accepted and scatters into grid_grad directly.        */
CJX_API int cjx_slice_ctf_loss_workspace_size(const cjx_slice_desc* desc, int64_t n_images,
                                              size_t* bytes);
/* Loss L_b = sum_pixels (simulate_b() - obs_b)^2 in real space (the
 * squared residual of the reference's README gradient example, with
 * padded_shape == shape) and its gradients, for every image b:
 *  - image_grads[b]: loss, dL/d(shift_x, shift_y, defocus) and dL/dR;
 *  - grid_grad (optional, complex64 N^3 in the reference's [z][y][x]
 *    layout): ACCUMULATES sum_b dL_b/dG by trilinear scatter-add (float2
 *    atomics), reported as dL/dRe + i dL/dIm (jax.grad returns the complex
 *    conjugate).  The caller zeroes it.
 * observed: device complex64 [n_images][Py][Px/2+1], rfftn of the observed
 * real-space images in cryoJAX's convention (ifftshift, then rfft2).
 * Resize path only, with N, Py, Px of the form 32 R (R in 1-6, 8, 10, 12, 16)
 * for the slice; on the Ewald sphere (CJX_EWALD_SPHERE, which needs
 * CJX_APPLY_CTF: the loss is on the contrast image) any size the forward
 * takes, on the shared-memory FFTs.
 * grid: C order, bricked, or x-pair bricked (16-byte aligned) for a voxel
 * grid; C order or bricked for spline coefficients.  grid_grad must be
 * 8-byte aligned (16 for the 16-byte atomics of CJX_TUNE_SCATTER_VEC 1).
 * Replaces jax.grad / eqx.filter_grad through LinearImageModel.simulate
 * (cryojax/simulator/_image_model/base_image_model.py:68-105, 297-328).      */
CJX_API int cjx_slice_ctf_loss_grad(const cjx_slice_desc* desc, const void* grid,
                                    const cjx_image_params* params, const int32_t* order,
                                    int64_t n_images, const void* observed,
                                    double* image_grads, void* grid_grad, void* workspace,
                                    size_t workspace_bytes, void* stream);

/* ---- orientation search ---------------------------------------------- */
typedef struct cjx_search_desc {
  cjx_slice_desc slice;          /* volume side, image shape, flags          */
  int64_t n_images;              /* observed images                          */
  int64_t n_orientations;        /* rows of the rotation table               */
  int32_t candidates_per_image;  /* K; 0 = every orientation (exhaustive)    */
  int32_t reserved;
} cjx_search_desc;

CJX_API int cjx_search_workspace_size(const cjx_search_desc* desc, size_t* bytes);
/* For every observed image b and each of its candidate orientations t
 * (candidates[b*K + k], or every t when candidates is NULL): simulate with
 * rotation rotations[t] (row-major 3x3 doubles) and image_params[b]'s CTF,
 * scale and shift (its rot field is ignored), score by normalised
 * cross-correlation against observed[b] (complex64 [Py][Px/2+1], rfftn of
 * the observed image), and keep the best.  Outputs: best_score[b],
 * best_orientation[b] (ties -> lowest index) and, when scores is non-NULL,
 * scores[b*K + k].  Replaces run_grid_search with MinimumSearchMethod over
 * an orientation grid whose fn simulates and scores
 * (cryojax/jax_util/_grid_search/search_loop.py:24-158).                    */
CJX_API int cjx_search(const cjx_search_desc* desc, const void* grid,
                       const cjx_image_params* image_params, const double* rotations,
                       const int32_t* candidates, const void* observed, float* scores,
                       float* best_score, int32_t* best_orientation, void* workspace,
                       size_t workspace_bytes, void* stream);

/* ---- several volumes / image shapes in one call ----------------------- */
typedef struct cjx_slice_group {
  cjx_slice_desc desc;             /* geometry and flags of this group        */
  const void* grid;                /* device, this group's volume             */
  const cjx_image_params* params;  /* device, n_images records                */
  const int32_t* order;            /* device processing order or NULL         */
  void* out;                       /* device complex64 [n_images][Py][Px/2+1] */
  int64_t n_images;
  int32_t tuning_valid;            /* 0: process defaults (cjx_tuning_set)     */
  int32_t gather_ilp;              /* 1, 2 or 4 when tuning_valid              */
  int32_t gather_tile;             /* 0, 1 or 2 when tuning_valid              */
  int32_t reserved;
} cjx_slice_group;

/* Workspace for cjx_slice_ctf_forward_multi: the largest group's need (the
 * groups run one after another on the stream and share it).                */
CJX_API int cjx_slice_ctf_multi_workspace_size(const cjx_slice_group* groups, int n_groups,
                                               size_t* bytes);
/* cjx_slice_ctf_forward for each group in turn on one stream, with per-group
 * kernel choices (from the autotuner).  All groups are validated before any
 * launch.  Replaces eqx.filter_vmap(simulate) over batches whose volumes and
 * image shapes differ, which the reference runs as separate traces.  The
 * whole call can be captured into one CUDA graph.                          */
CJX_API int cjx_slice_ctf_forward_multi(const cjx_slice_group* groups, int n_groups,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free variant of cjx_slice_ctf_forward.  No counterpart in the
 * reference.  For callers that cannot allocate device memory, because the
 * runtime hosting them owns every allocation (for example an XLA custom call
 * without a scratch allocator) or forbids allocation once it is running: the
 * caller passes only inputs and outputs, and the resize stage's scratch is a
 * fixed array of CJX_NOALLOC_SCRATCH_BYTES inside the library, held by every
 * GPU that loads the library until the process exits.  Results equal
 * cjx_slice_ctf_forward's.
 *  - The first call on each device looks up that array's device address;
 *    make that first call before any stream capture.  The address is cached
 *    for the life of the process and does not survive a reset of the
 *    device (cudaDeviceReset): do not call this again on a reset device.
 *  - All calls on a device share the array: calls that overlap on the GPU
 *    (other streams, other host threads) race; serialise them.
 *  - Returns CJX_ERR_UNSUPPORTED if one image, or desc->images_per_chunk
 *    images, need more scratch than CJX_NOALLOC_SCRATCH_BYTES.
 *  - Calls no cudaMalloc / cudaFree or any allocating library routine.      */
#define CJX_NOALLOC_SCRATCH_BYTES (32u << 20)
CJX_API int cjx_slice_ctf_forward_noalloc(const cjx_slice_desc* desc, const void* grid,
                                          const cjx_image_params* params, const int32_t* order,
                                          int64_t n_images, void* out, void* stream);

/* Bricked volume layout (no counterpart in the reference; a device-side
 * re-layout of FourierVoxelGridVolume.fourier_voxel_grid, or of a
 * FourierVoxelSplineVolume's coefficients with n = N + 2).  8x8x8 blocks in
 * C order; inside a block the voxels are in Morton order, so every 2x2x2
 * brick is 64 contiguous bytes.  A slice plane at any orientation then reads
 * compact voxel clusters per DRAM burst.  Sides are padded to a multiple of
 * 8 with zeros (never read: indices >= N are out of bounds).
 * cjx_bricked_volume_size: bytes of the bricked copy of an N^3 grid.
 * cjx_brick_volume: write it (stream-ordered; grid and bricked distinct).  */
CJX_API int cjx_bricked_volume_size(int n, size_t* bytes);
CJX_API int cjx_brick_volume(int n, const void* grid, void* bricked, void* stream);
/* The x-pair copy (CJX_GRID_BRICKED_PAIRS): twice cjx_bricked_volume_size
 * bytes; entry (x, y, z) = (g(x, y, z), g(x+1, y, z)), zero past the edge.
 * n may be up to CJX_MAX_SIDE + 2 (a spline coefficient array's side).      */
CJX_API int cjx_brick_volume_pairs(int n, const void* grid, void* pairs, void* stream);

/* Cubic-spline coefficients of a centred Fourier voxel grid: `grid` N^3
 * complex64 (C order) -> `coefficients` (N + 2)^3 complex64 (C order).
 * Replaces compute_spline_coefficients
 * (cryojax/ndimage/_map_coordinates.py:71-82, 179-215) as called by
 * FourierVoxelSplineVolume.from_real_voxel_grid
 * (cryojax/simulator/_volume/representations/voxel_volume.py:163-203):
 * along x, then y, then z, each line of length L gets c2 = d[0]/6,
 * c_{L+1} = d[L-1]/6, the tridiag(1, 4, 1) solve for the interior and the
 * two end extrapolations.  Solved in double precision, stored complex64.
 * N in [4, CJX_MAX_SIDE]; grid and coefficients distinct; scratch of
 * cjx_spline_coefficients_workspace_size bytes (N (N + 2)^2 complex64).
 * Stream-ordered.                                                          */
CJX_API int cjx_spline_coefficients_workspace_size(int n, size_t* bytes);
CJX_API int cjx_spline_coefficients(int n, const void* grid, void* coefficients, void* workspace,
                                    size_t workspace_bytes, void* stream);

/* ---- Gaussian-mixture rendering ----------------------------------------
 * GaussianMixtureRenderFn (cryojax/simulator/_volume_rendering/
 * gaussian_rendering.py:24-336) for a GaussianMixtureVolume
 * (cryojax/simulator/_volume/representations/gaussian_volume.py:21-180):
 * grid[z][y][x] (float32, device) = sum over atoms and their Gaussians of
 * amplitude / (2 dx)^3 times, per axis, erf(s (L - p + dx)) - erf(s (L - p)),
 * s = 1 / sqrt(2 variance), L = (i - D/2) dx - dx/2.  positions [n][3]
 * (x, y, z, Angstrom), amplitudes and variances [n][n_gaussians] (variances
 * in Angstrom^2, positive), all float32 device arrays.  Each atom adds to
 * the voxels within cutoff_sigmas standard deviations (plus one voxel) of
 * it (0 = the default 7), with float atomics (summation order varies run
 * to run at rounding level).  The grid is zeroed first unless
 * CJX_RENDER_ACCUMULATE.  Stream-ordered.                                   */
#define CJX_RENDER_ACCUMULATE 1u
#define CJX_RENDER_MAX_GAUSSIANS 8
typedef struct cjx_render_desc {
  int32_t nz, ny, nx;        /* grid shape                                  */
  int32_t n_gaussians;       /* per atom, 1..CJX_RENDER_MAX_GAUSSIANS       */
  float voxel_size;          /* Angstrom                                    */
  float cutoff_sigmas;       /* 0 = default (7)                              */
  uint32_t flags;            /* CJX_RENDER_*                                */
  int32_t reserved;
} cjx_render_desc;
CJX_API int cjx_render_gaussians(const cjx_render_desc* desc, const float* positions, const float* amplitudes,
                                 const float* variances, int64_t n_atoms, float* grid, void* stream);

/* Batched complex-to-complex FFTs of `count` contiguous rows of n complex64
 * values (direction -1: forward, numpy.fft.fft; +1: unnormalised inverse,
 * n * numpy.fft.ifft), with the same warp FFTs the resize stage uses.  No
 * counterpart in the reference (which calls jnp.fft); a utility and test
 * hook.  in and out must not alias.                                        */
CJX_API int cjx_fft_c2c(int n, int direction, const void* in, void* out, int64_t count,
                        void* stream);

/* ---- real-space output and post-processing ---------------------------- */
/* AbstractImageModel.postprocess after the Fourier image
 * (cryojax/simulator/_image_model/base_image_model.py:107-158): for each
 * image b, out[b] (float32 [h][w]) = mask * normalise(crop(irfftn(
 * fourier[b], s=(py, px)))), where
 *  - irfftn is cryoJAX's (cryojax/ndimage/_fft.py:57-77): inverse real FFT
 *    of the rfft half plane complex64 [py][px/2+1] (zero frequency in the
 *    corner), scaled by 1 / (py px), then fftshift; the kx = 0 and (even px)
 *    kx = px/2 columns count only with their Hermitian part in ky, as an
 *    inverse real FFT reads them;
 *  - crop is the centre crop to (h, w) <= (py, px)
 *    (cryojax/ndimage/_edges.py:15-62), a no-op when equal;
 *  - with CJX_PP_NORMALIZE: (x - mean) / std over the h w pixels, the
 *    population std (cryojax/ndimage/_normalize.py:11-28);
 *  - mask: optional float32 [h][w] multiplied in last (NULL: none).
 * workspace: at least cjx_postprocess_workspace_size(1, ...) bytes; a
 * larger one lets more images share a pass.  Stream-ordered.              */
#define CJX_PP_NORMALIZE 1u
CJX_API int cjx_postprocess_workspace_size(int64_t n_images, int py, int px, size_t* bytes);
CJX_API int cjx_postprocess_real(int64_t n_images, int py, int px, int h, int w, uint32_t flags,
                                 const void* fourier, const float* mask, float* out, void* workspace,
                                 size_t workspace_bytes, void* stream);
/* cryoJAX's rfftn of real-space images (cryojax/ndimage/_fft.py:80-99):
 * out[b] (complex64 [py][px/2+1]) = rfft2(ifftshift(image[b])), image
 * float32 [n][py][px].  Used for observed images and for post-processed
 * images whose Fourier form is requested.  Needs no workspace; image and
 * out must not overlap.  Stream-ordered.                                   */
CJX_API int cjx_rfft2(int64_t n_images, int py, int px, const float* image, void* out, void* stream);

/* Process-wide tuning knobs (no counterpart in the reference; set by the
 * autotuner).  CJX_TUNE_GATHER_ILP: samples whose corner loads one lane
 * issues together in the gather (1, 2 or 4).  CJX_TUNE_CHUNK_BYTES: target
 * workspace bytes per chunk when desc->images_per_chunk is 0 (default 2 GiB).
 * CJX_TUNE_GATHER_MODE: 1 = separate gather kernel (no shared memory) and
 * column-FFT kernel, 0 = one fused gather + column-FFT kernel with
 * shared-memory FFTs (C-order and bricked grids only), 2 (default) = one
 * fused gather + register-FFT column kernel (trilinear grids in any layout,
 * slice or Ewald sphere, N = 32 R; other cases, e.g. spline volumes, run
 * as 1), which never writes the sampled plane to memory.
 * CJX_TUNE_FFT_MODE: 1 = register/shuffle FFTs where the length is 32 R
 * (R in 1-6, 8, 10, 12, 16), 2 = the same, with the 512-point
 * column transforms of the resize stage done as 16 x 32 through one
 * shared-memory transpose instead of five shuffle stages, 3 (default) = as
 * 2 and the row pass's 512-point inverse transforms the same way, 0 = shared-memory
 * Stockham FFTs everywhere.
 * CJX_TUNE_GATHER_TILE: lanes of a gather warp cover 2 x 16 (0), 4 x 8 (1)
 * or 8 x 4 (2) samples (columns x rows) of the slice plane; 3 = one column
 * x 32 rows in gather mode 2 (the split gather takes 3 as 0).
 * CJX_TUNE_SCATTER_VEC: how the adjoint's grid scatter-add issues its
 * atomics.  1 (default) = the two x-corners of a corner row in one 16-byte
 * atomic when they are adjacent and 16-byte aligned (even x0), else two
 * 8-byte atomics (a grid_grad that is only 8-byte aligned takes 0); 0 = one
 * 8-byte atomic per (sample, corner); 2 = warp-aggregated: lanes whose
 * corner lands on the same voxel sum their contributions with warp shuffles
 * and one lane per voxel issues the atomic.
 * CJX_TUNE_SPLINE_ILP: samples per lane in the cubic-spline gather
 * (CJX_GRID_SPLINE; 1, 2 or 4, default 4).                                 */
#define CJX_TUNE_GATHER_ILP 1
#define CJX_TUNE_CHUNK_BYTES 2
#define CJX_TUNE_GATHER_MODE 3
#define CJX_TUNE_FFT_MODE 4
#define CJX_TUNE_GATHER_TILE 5
#define CJX_TUNE_SCATTER_VEC 6
#define CJX_TUNE_SPLINE_ILP 7
/* CJX_TUNE_MULTI_WAVES: 1 = cjx_slice_ctf_forward_multi runs its groups in
 * waves, each wave holding a slice of every group's images and each pass
 * of the resize path launched once for all groups (so small and large
 * groups share every launch), when every group takes the fused
 * register-FFT path (gather mode 2, trilinear slice, resize, sizes 32 R, one
 * grid layout); the group records' gather choices are then not used.
 * 0 = the groups one after another.                                         */
#define CJX_TUNE_MULTI_WAVES 9
CJX_API int cjx_tuning_set(int key, int64_t value);
CJX_API int cjx_tuning_get(int key, int64_t* value);

/* Measurement helper: streams `bytes` of `buf` `passes` times through the
 * SMs (read-only, 16-byte vector loads, result folded into `sink`).  With a
 * buffer smaller than L2 this measures L2 read bandwidth; larger, HBM.
 * No counterpart in the reference (roofline denominator).                  */
CJX_API int cjx_probe_read_bandwidth(const void* buf, size_t bytes, int passes,
                             void* sink, void* stream);

/* Measurement helpers (no counterpart in the reference).  While enabled on
 * the calling thread, each kernel launch the library makes is bracketed by
 * a pair of CUDA events on its stream.  cjx_profile_read waits for those
 * events, then writes up to max_kernels entries: kernel name (32 chars,
 * NUL-padded, into names[32*i]), launch count and summed milliseconds; it
 * clears the record.                                                       */
CJX_API int cjx_profile_enable(int on);
CJX_API int cjx_profile_read(char* names, int64_t* counts, double* total_ms,
                             int max_kernels, int* n_kernels);

/* ---- template-sharing exhaustive search --------------------------------- */
/* The NCC of every (image, orientation) pair from two FP16 tensor-core
 * GEMMs (cjx_gemm with CJX_GEMM_F16): num = Y S^T over K = 2 Py (Px/2+1)
 * and den = Z P^T over K = Py (Px/2+1), where S_t is the CTF-free slice of
 * orientation t (Hermitian-fixed columns), P_t = |S_t|^2, Y_b = w conj(m_b)
 * O_b and Z_b = w |m_b|^2 (m_b: image b's CTF, envelope, translation and
 * scale; w: Parseval weights, 0 at DC).  Rows are FP16 at unit RMS; Py must
 * be a multiple of 8 (the rows are the GEMM operands).  No counterpart in
 * the reference (its grid search simulates every pair).                    */
/* images: complex64 [n][Py][Px/2+1] CTF-free slices -> s16 [n][2 Py (Px/2+1)],
 * p16 [n][Py (Px/2+1)] (FP16).                                             */
CJX_API int cjx_pack_templates(const void* images, int64_t n, int py, int px, void* s16,
                               void* p16, void* stream);
/* observed: complex64 [n][Py][Px/2+1] (rfftn of the observed images);
 * params: the images' records (rotation ignored); flags: the CJX_APPLY_*
 * bits of the image model -> y16, z16 (FP16 rows), oo = sum w |O|^2 and
 * the rows' RMS scales yinv, zinv.                                         */
CJX_API int cjx_pack_observed(const void* observed, const cjx_image_params* params, int64_t n,
                              int py, int px, int flags, void* y16, void* z16, float* oo,
                              float* yinv, float* zinv, void* stream);
/* NCC(b, t0 + t) = num[b][t] yinv[b] / sqrt(den[b][t] zinv[b] oo[b]) for t
 * in [0, T) (num, den: FP32 [n][ld]); writes scores[b][t0 + t] when scores
 * is non-NULL and the row's best (ties -> lowest index) into best_score /
 * best_orientation, or merges it with their current values when
 * accumulate_best != 0 (orientation blocks processed in increasing t0).    */
CJX_API int cjx_ncc_argmax(const float* num, const float* den, int64_t ld, int64_t n, int64_t T,
                           const float* oo, const float* yinv, const float* zinv, int64_t t0,
                           float* scores, int64_t ld_scores, float* best_score,
                           int32_t* best_orientation, int accumulate_best, void* stream);

/* The k <= 16 highest NCCs of each row (same formula as cjx_ncc_argmax) as
 * template indices, descending, ties -> lower index: indices[b][0..k).
 * Rescoring them with cjx_search (candidate lists, FP32) makes the
 * template-sharing search's answer exact whenever the FP32 optimum is among
 * them.                                                                    */
CJX_API int cjx_ncc_topk(const float* num, const float* den, int64_t ld, int64_t n, int64_t T,
                         const float* oo, const float* yinv, const float* zinv, int k,
                         int32_t* indices, void* stream);

/* FP32 re-ranking from a bank of the templates' FP32 simulations instead
 * of simulating each candidate again.  cjx_pack_observed32 writes each
 * image's unscaled FP32 terms y32 = w conj(m) O (complex64 [n][Py][Px/2+1]),
 * z32 = w |m|^2 (float [n][Py][Px/2+1]) and oo = sum w |O|^2 (same w and m
 * as cjx_pack_observed).  cjx_ncc_rerank32 scores image b against its m
 * <= 16 candidates candidates[b][0..m) from bank (complex64 [T][Py][Px/2+1],
 * the CTF-free simulations cjx_pack_templates packs):
 *   NCC = sum y32 . S / sqrt(sum z32 |S|^2 * oo)
 * with S the Hermitian-fixed template, FP32 sums (-inf for an index outside
 * [0, T)); the best (ties -> lower index) goes to best_score /
 * best_orientation and every NCC to scores[b][0..m) when scores is not
 * NULL.  The same NCC as the simulating scorer's up to FP32 rounding.      */
CJX_API int cjx_pack_observed32(const void* observed, const cjx_image_params* params, int64_t n,
                                int py, int px, int flags, void* y32, float* z32, float* oo,
                                void* stream);
CJX_API int cjx_ncc_rerank32(const void* bank, int py, int px, int64_t T, const void* y32,
                             const float* z32, const float* oo, int64_t n,
                             const int32_t* candidates, int m, float* scores, float* best_score,
                             int32_t* best_orientation, void* stream);

/* The learned search's rescoring from the same template rows: for image b
 * and proposed-direction slot k (dirs [n][kd], int32), the n_inplane
 * templates t = dirs[b][k] n_inplane + a (a in [0, n_inplane)) give
 *   num[b][k n_inplane + a] = y16[b] . s16[t] (K = 2 kp),
 *   den[b][k n_inplane + a] = z16[b] . p16[t] (K = kp),
 * the inputs of cjx_ncc_argmax / cjx_ncc_topk over kd n_inplane columns
 * (kp = Py (Px/2+1), a multiple of 8; rows 16-byte aligned; s16 / p16
 * hold n_dir n_inplane rows).  The (image, slot) pairs are sorted by
 * direction and taken 16 at a time with that direction's templates: FP16
 * products, FP32 sums on the tensor cores (mma.sync m16n8k16), each
 * template row read once per 16 pairs.  A direction outside [0, n_dir)
 * gives zero sums.  workspace:
 * cjx_ncc_directions_workspace_size bytes.  No counterpart in the reference
 * (its search simulates every candidate).                                   */
CJX_API int cjx_ncc_directions_workspace_size(int64_t n, int kd, int n_dir, size_t* bytes);
CJX_API int cjx_ncc_directions(const void* y16, const void* z16, const void* s16, const void* p16, int64_t n,
                               int64_t kp, const int32_t* dirs, int kd, int n_dir, int n_inplane, float* num,
                               float* den, void* workspace, size_t workspace_bytes, void* stream);

/* ---- tensor-core GEMM (pose-proposal network) -------------------------- */
#define CJX_GEMM_OUT_BF16 1   /* store C as BF16 (default FP32)              */
#define CJX_GEMM_BIAS 2       /* C[:, n] += bias[n] (FP32)                    */
#define CJX_GEMM_RELU 4       /* C = max(C, 0) after the bias                 */
#define CJX_GEMM_ACCUMULATE 8 /* C += A B^T with FP32 atomics (split_k > 1)   */
#define CJX_GEMM_F16 16       /* A and B are FP16 (default BF16)              */
/* C[M][ldc] = A B^T for A [M][lda], B [N][ldb] (16-bit, K-major; base
 * 16-byte aligned, lda and ldb multiples of 8 elements), FP32 accumulation
 * on the tensor cores (tcgen05.mma, accumulator in tensor memory, operands
 * staged by TMA).  split_k > 1 splits the K loop over CTAs and needs
 * CJX_GEMM_ACCUMULATE.  The network's layers are implicit GEMMs over
 * these.  No counterpart in the reference (its pose search has no network).
 * Kernels that give up on a wait (2 s limit) record a code readable with
 * cjx_device_status.                                                       */
CJX_API int cjx_gemm(int64_t M, int64_t N, int64_t K, const void* A, int64_t lda,
                     const void* B, int64_t ldb, void* C, int64_t ldc,
                     const float* bias, int flags, int split_k, void* stream);
/* First error code recorded by a device-side wait that gave up (0 = none);
 * synchronises `stream`; reset != 0 clears it.                             */
CJX_API int cjx_device_status(int* status, int reset, void* stream);
/* Failure-path self-test of the tensor-core kernels' bounded waits: one
 * thread waits on an mbarrier that nothing arrives on; after limit_ns
 * (1 us .. 2 s) the wait gives up and writes 105 into *device_status (a
 * device int the caller zeroed) if it is still 0.  The kernel returns
 * normally; the context stays usable.                                      */
CJX_API int cjx_selftest_bounded_wait(uint64_t limit_ns, int* device_status, void* stream);

/* ---- pose-proposal network kernels (no counterpart in the reference) --- */
/* Activations are NHWC BF16; a 3x3 stride-2 pad-1 convolution is
 * im2col -> cjx_gemm (bias + ReLU fused) and its backward is cjx_gemm ->
 * cjx_cnn_col2im.  Sizes are in elements.                                  */

/* out[b] (BF16 [h][w]) = (x - mean) / std of x = images[index ? index[b] : b]
 * + sigma_b * N(0, 1), sigma_b^2 = var(images[.]) / snr; snr <= 0 adds no
 * noise.  The normal draws are a counter-based function of (seed, source
 * image, pixel).                                                           */
CJX_API int cjx_cnn_noisy_normalize(const float* images, const int64_t* index, int64_t n,
                                    int h, int w, float snr, uint64_t seed, void* out,
                                    void* stream);
/* dst[b] (FP32 [h][w]) = area-weighted mean of src[b] (FP32 [H][W]) over
 * each output pixel's footprint (H/h x W/w input pixels, fractional overlaps
 * weighted): the network's input size from any observed image size.        */
CJX_API int cjx_area_downsample(const float* src, int64_t n, int H, int W, float* dst, int h,
                                int w, void* stream);
/* col[p][k] (BF16, row pitch ldk >= 9C, ldk % 8 == 0) of x [B][H][W][C]:
 * p = (b H/2 + oy) W/2 + ox, k = (3 ky + kx) C + c, zeros in [9C, ldk).    */
CJX_API int cjx_cnn_im2col(const void* x, int64_t B, int H, int W, int C, void* col,
                           int64_t ldk, void* stream);
/* The first layer at inference without the im2col matrix: y (BF16
 * [B][H/2][W/2][cout], 16-byte aligned) = ReLU(conv3x3_s2(x) + bias) for a
 * one-channel BF16 x [B][H][W], weights w (BF16 [cout][ldk], tap k = 3 ky +
 * kx) and FP32 bias (may be NULL); cout = 32.  What cjx_cnn_im2col and the
 * tensor-core GEMM give for that layer, summed in tap order.               */
CJX_API int cjx_cnn_conv0(const void* x, int64_t B, int H, int W, const void* w, int64_t ldk,
                          int cout, const float* bias, void* y, void* stream);
/* The later layers at inference without the im2col matrix (implicit GEMM
 * on the tensor cores, mma.sync m16n8k16 BF16 with FP32 accumulation): y
 * (BF16 NHWC [B][H/2][W/2][cout]) = ReLU(conv3x3_s2(x) + bias) for x (BF16
 * NHWC [B][H][W][C], 16-byte aligned), weights w (BF16 [cout][ldk], k =
 * (3 ky + kx) C + c, the cjx_cnn_im2col order) and FP32 bias (may be NULL);
 * (C, cout) in (32, 64), (64, 128), (128, 128), (128, 256), (256, 256).    */
CJX_API int cjx_cnn_conv_s2(const void* x, int64_t B, int H, int W, int C, const void* w,
                            int64_t ldk, int cout, const float* bias, void* y, void* stream);
/* dx (BF16 [B][H][W][C]) = col2im(dcol) (FP32 [p][ldk]), multiplied by
 * (act > 0) when act (BF16, same shape as dx) is non-NULL.                 */
CJX_API int cjx_cnn_col2im(const float* dcol, int64_t ldk, const void* act, int64_t B, int H,
                           int W, int C, void* dx, void* stream);
/* out[c][r] (BF16, pitch ld_out) = in[r][c] (FP32 or BF16, pitch ld_in).   */
CJX_API int cjx_transpose_to_bf16(const void* in, int in_is_bf16, int64_t rows, int64_t cols,
                                  int64_t ld_in, void* out, int64_t ld_out, void* stream);
/* out[i] (BF16) = grad[i] * (act == NULL || act[i] > 0).                   */
CJX_API int cjx_relu_mask(const float* grad, const void* act, int64_t n, void* out,
                          void* stream);
/* out[c] += sum_r x[r][c] (FP32 atomics; the caller zeroes out).          */
CJX_API int cjx_colsum(const void* x, int x_is_bf16, int64_t rows, int64_t cols, int64_t ld,
                       float* out, void* stream);
/* Softmax cross entropy per row of logits [B][C] against the target
 * (1 - smoothing) at labels[r] plus smoothing spread evenly over the
 * n_neighbours entries neighbours[labels[r]][.] (over all C classes when
 * neighbours is NULL).  loss[r] (optional) and dlogits (BF16 [B][C],
 * optional) = (softmax - target) * grad_scale.                             */
CJX_API int cjx_softmax_xent(const float* logits, int64_t B, int C, const int32_t* labels,
                             const int32_t* neighbours, int n_neighbours, float smoothing,
                             float grad_scale, float* loss, void* dlogits, void* stream);
typedef struct cjx_param_segment {
  int64_t offset;       /* first element in the flat parameter vector       */
  int64_t count;        /* elements                                         */
  int64_t cols;         /* > 0: a weight stored [count/cols][cols] (K x out) */
  int64_t ldk;          /* row pitch of w_bf16 (>= count / cols)            */
  void* w_bf16;         /* optional BF16 copy [cols][ldk] (out x K)         */
  void* wt_bf16;        /* optional BF16 copy [count/cols][cols]            */
  int32_t weight_decay; /* 1: apply decoupled weight decay                  */
  int32_t reserved;
} cjx_param_segment;
/* AdamW step `step` (>= 1) over the flat FP32 vector params (n elements)
 * with gradients grads and moments m, v; refreshes the weight segments'
 * BF16 copies.  Segments are sorted by offset, the first at 0, <= 24.     */
CJX_API int cjx_adamw(float* params, const float* grads, float* m, float* v, int64_t n,
                      const cjx_param_segment* segments, int n_segments, float lr, float beta1,
                      float beta2, float eps, float weight_decay, int64_t step, void* stream);
/* Per row of logits [B][C] (C <= 1024): the k largest (ties -> lower
 * index) into dirs[B][k] (optional) and candidates[B][k * n_inplane] =
 * dirs * n_inplane + a for a in [0, n_inplane) (optional).                 */
CJX_API int cjx_topk_candidates(const float* logits, int64_t B, int C, int k, int n_inplane,
                                int32_t* dirs, int32_t* candidates, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CRYOJAX_B200_H */
