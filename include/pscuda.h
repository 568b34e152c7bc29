/*
 * libpscuda -- C ABI of the B200 (sm_100a) implementation of PolySpec's
 * data-parallel hot path: HEALPix spin-0/spin-s spherical harmonic
 * transforms, pixel-space products and radial sums, and the vector kernels of
 * the masked conjugate-gradient S^-1 filter.
 *
 * Conventions
 *  - Every entry point returns 0 on success or a negative PS_ERR_* code; no
 *    C++ exception crosses the ABI.  ps_error_string() names a code.
 *  - Every data pointer is a device pointer owned by the caller.  Plans own
 *    only their read-only tables (ring geometry, Legendre seeds, FFT tables);
 *    a plan is immutable after ps_plan_create and may be shared by callers
 *    on different streams.  Scratch memory is passed in explicitly
 *    (ps_*_workspace_bytes gives the size), so no call allocates.
 *  - Work is enqueued on the given stream; nothing synchronises the host.
 *  - Layouts (as in the reference and ducc0): alm are complex128 (re, im
 *    interleaved) in the HEALPix m-major order idx = m(2 lmax + 1 - m)/2 + l
 *    with mmax = lmax; maps are float64 in RING order.  Spin 0 works on
 *    alm[batch][nalm] <-> map[batch][npix]; spin s > 0 on
 *    alm[batch][2][nalm] (G, C) <-> map[batch][2][npix] (Q, U).
 */
#ifndef PSCUDA_H
#define PSCUDA_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PS_OK = 0,
  PS_ERR_INVALID = -1,      /* bad argument (size, spin, null pointer) */
  PS_ERR_UNSUPPORTED = -2,  /* valid but not supported by this build */
  PS_ERR_NOMEM = -3,        /* table allocation at plan creation failed */
  PS_ERR_CUDA = -4,         /* a CUDA runtime call or launch failed */
  PS_ERR_WORKSPACE = -5,    /* workspace too small */
  PS_ERR_NOT_CONVERGED = -6 /* iterative solver hit its step limit */
};

enum { PS_PREC_FP64 = 0, PS_PREC_MIXED = 1 };

typedef struct ps_plan ps_plan;

const char* ps_error_string(int code);
int ps_version(void);
int ps_device_sm_count(int* count);

/* ----------------------------------------------------------------- SHT plans
 * Replaces the geometry/setup the reference takes from
 * ducc0.healpix.Healpix_Base(Nside, "RING").sht_info()  (polyspec/base.py:70-74).
 * spin_mask: bit s set => seeds for spin s are built (bit 0 = spin 0).
 */
int ps_plan_create(int nside, int lmax, int mmax, int spin_mask, int prec, ps_plan** plan);
int ps_plan_destroy(ps_plan* plan);
int ps_plan_info(const ps_plan* plan, int* nside, int* lmax, int64_t* npix, int64_t* nalm);
/* Device error flag of the plan: kernels set it when a bounded wait expires
 * (they then return without completing).  Reads it (synchronously, after the
 * device finishes its work) and optionally clears it.  No reference counterpart. */
int ps_plan_error_flag(const ps_plan* plan, int* value, int reset);

/* prec = PS_PREC_FP64: every stage in FP64.  prec = PS_PREC_MIXED: the
 * synthesis' Legendre stage runs on the tensor cores (tcgen05, TF32 split in
 * three products, FP32 accumulation) from FP64 recurrences; the adjoint's
 * Legendre stage contracts FP32-rounded FP64 recurrences with FP32 FMAs; the
 * ring transforms run in FP32; inputs and outputs stay FP64 in both cases. */

/* Scratch bytes needed by ps_synthesis / ps_adjoint for `batch` maps of `spin`. */
int ps_sht_workspace_bytes(const ps_plan* plan, int batch, int spin, int adjoint, size_t* bytes);

/* alm -> map.  Replaces ducc0.sht.synthesis(alm=..., lmax, spin, mmax=lmax,
 * theta_interpol=False, **ducc_geom) as called at polyspec/base.py:172-176
 * (to_map), :225 and :230-231 (to_map_vec) and :282 (to_map_spin). */
int ps_synthesis(const ps_plan* plan, const double* alm, double* map, int batch, int spin,
                 void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* map -> alm, scaled by `scale` (the reference uses pi/(3 nside^2) = 4 pi/Npix).
 * Replaces ducc0.sht.adjoint_synthesis(...) * pi/(3 Nside^2) at
 * polyspec/base.py:147-151 (to_lm), :193 and :206 (to_lm_vec), :253 (to_lm_spin). */
int ps_adjoint(const ps_plan* plan, const double* map, double* alm, int batch, int spin, double scale,
               void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* Allocation-free variant of ps_synthesis (no counterpart in the reference).
 * For callers that cannot allocate device memory at the point of the call (a
 * framework that owns all device memory through its own fixed allocator, a
 * real-time loop where a synchronising cudaMalloc is not allowed): the scratch
 * comes from a static device array of PS_NOALLOC_SCRATCH_BYTES held by every GPU
 * that loads the library until exit.  Requests needing more scratch than that
 * (ps_sht_workspace_bytes) return PS_ERR_WORKSPACE before anything runs.  The
 * first call on a device looks up the array's address and should come before
 * any stream capture.  Calls share the array: calls that overlap on the GPU race. */
#define PS_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int ps_synthesis_noalloc(const ps_plan* plan, const double* alm, double* map, int batch, int spin,
                         cudaStream_t stream);

/* ------------------------------------------------------------- launch statistics
 * No reference counterpart beyond its wall-clock SHT timer (polyspec/base.py:113-127,
 * polyspec/tspec_template.py:453-517): every kernel launch of the library is
 * counted per kind with its algorithmic flops and bytes; with timing enabled,
 * CUDA events bracket each launch and ps_stats_get returns the summed device
 * time (it synchronises on those events). */
enum {
  PS_K_LEG_SYNTH = 0,   /* Legendre stage of synthesis (all spins) */
  PS_K_LEG_ADJOINT = 1, /* Legendre stage of the adjoint */
  PS_K_FFT_SYNTH = 2,   /* ring transforms of synthesis */
  PS_K_FFT_ADJOINT = 3, /* ring transforms of the adjoint */
  PS_K_LAYOUT = 4,      /* alm transposes and partial-sum reductions */
  PS_K_PIXEL = 5,       /* pixel-space products and sums */
  PS_K_VECTOR = 6,      /* harmonic-space vector kernels (CG, filters) */
  PS_K_MLP = 7,         /* learned-preconditioner network */
  PS_KERNEL_KINDS = 8
};
int ps_stats_enable_timing(int on);
int ps_stats_reset(void);
int ps_stats_get(int kind, int64_t* launches, double* ms, double* flops, double* bytes);

#ifdef __cplusplus
}
#endif

#endif /* PSCUDA_H */
