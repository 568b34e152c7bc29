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
 *    apart from its tile setting (ps_plan_set_tile) a plan is immutable after
 *    ps_plan_create and may be shared by callers on different streams.  Scratch memory is passed in explicitly
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

/* Tile setting of the Legendre stages (no reference counterpart): maps per CTA
 * for direction 0 (synthesis) or 1 (adjoint) and one spin; 0 restores the
 * library's choice by batch size.  Allowed: mixed synthesis spin 0 {8, 16, 32},
 * spin s {4, 8}; mixed adjoint spin 0 {1, 8}, spin s {1, 4}; FP64 synthesis
 * spin 0 {1, 4}, spin s {1, 2}; FP64 adjoint spin 0 {1, 4}, spin s {1}
 * (PS_ERR_UNSUPPORTED otherwise).  Used by the autotuner; it changes the plan,
 * so it must not run concurrently with transforms on the same plan. */
int ps_plan_set_tile(ps_plan* plan, int direction, int spin, int tile);

/* prec = PS_PREC_FP64: every stage in FP64.  prec = PS_PREC_MIXED: the
 * synthesis' Legendre stage runs on the tensor cores (tcgen05, TF32 split in
 * three products, FP32 accumulation) from FP64 recurrences; the adjoint's
 * Legendre stage contracts FP32-rounded FP64 recurrences with FP32 FMAs; the
 * ring transforms run in FP32; inputs and outputs stay FP64 in both cases.
 *
 * Legendre tables (mixed plans only; no reference counterpart -- ducc0 always
 * recomputes the recurrences).  ps_plan_build_table computes the FP32 Legendre
 * values of one spin once (FP64 recurrence, as the on-the-fly kernels) into a
 * table the plan owns (ps_plan_table_bytes: Rh * nalm * 4 bytes for spin 0,
 * twice that for spin s, Rh = 2 nside rounded up to 128; 17.7 GB and 35.4 GB
 * at nside 1024, lmax 2048).  From then on both Legendre stages of that spin
 * -- on the plan and on its band plans -- are streaming tensor-core GEMMs over
 * the table (TF32 split in three products, FP32 sums), and the adjoint writes
 * alm without per-ring-tile partial sums (its workspace shrinks: query
 * ps_sht_workspace_bytes after building).  The build allocates (cudaMalloc)
 * and enqueues on `stream`; it returns PS_ERR_NOMEM when the table does not
 * fit, PS_ERR_UNSUPPORTED on FP64 or band plans.  ps_plan_drop_tables frees
 * them (after synchronising the device); ps_plan_has_table tells whether a
 * spin's transforms use one. */
/* Table format of the tables a plan builds next (tables already built keep theirs):
 * PS_TAB_TF32X3 -- FP32 values, split into TF32 hi + lo by the GEMM kernels (3 products);
 * PS_TAB_BF16X3 -- the same FP32 values stored as BF16 hi + mid + lo planes (24 significant
 * bits) already in the tensor core's operand layout, 1.5x the bytes, streamed into the MMAs
 * by bulk copies with no operand splitting (kind::f16, 6 products). */
enum { PS_TAB_TF32X3 = 0, PS_TAB_BF16X3 = 1 };
int ps_plan_set_table_format(ps_plan* plan, int format);
int ps_plan_table_bytes(const ps_plan* plan, int spin, size_t* bytes);
int ps_plan_build_table(ps_plan* plan, int spin, cudaStream_t stream);
int ps_plan_has_table(const ps_plan* plan, int spin, int* has);
int ps_plan_drop_tables(ps_plan* plan);

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

/* Fused weighted round trip of the masked CG operator (no single reference call;
 * replaces, per spin, the pair to_map -> pixel weight -> to_lm inside
 * CGD._apply_A at polyspec/weighting.py:297-299):
 *   alm_out[b] = scale * lscale * Y^H W Y (lscale * alm_in[b])
 * with Y this plan's synthesis of `spin`, W = weight [ncomp][npix] (float64;
 * spin 0: one component; spin s: Q and U), lscale [ncomp][nalm] (float64, e.g.
 * the beam per lm; NULL = 1).  alm element (b, c, idx) is at
 * alm[b * alm_stride + c * nalm + idx] (complex128; alm_stride >= ncomp * nalm
 * complex elements, so T and (E, B) of a [batch][3][nalm] array are used in
 * place).  Needs a mixed plan holding the Legendre table of `spin`
 * (ps_plan_build_table); PS_ERR_UNSUPPORTED otherwise.  The maps are never
 * written to memory: each ring is synthesised, weighted and transformed back
 * in shared memory.  alm_in and alm_out must not overlap. */
int ps_roundtrip_workspace_bytes(const ps_plan* plan, int batch, int spin, size_t* bytes);
int ps_sht_weighted_roundtrip(const ps_plan* plan, const double* alm_in, double* alm_out, int64_t alm_stride,
                              int batch, int spin, const double* weight, const double* lscale, double scale,
                              void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* Legendre stages alone (no reference counterpart; ducc0 exposes the same split
 * as its leg2alm / alm2leg), in the plan's precision (a mixed plan converts the
 * phases to complex64 internally; inputs and outputs stay complex128):
 *   ps_legendre_synthesis  alm [batch][ncomp][nalm] -> phase [R][mmax+1][batch][ncomp]
 *   ps_legendre_adjoint    phase -> alm (times scale), the exact adjoint
 * where phase holds, for every ring and order m, the m-th Fourier coefficient
 * of the ring (complex128; for spin s the pair Q, U).  Used on a ring-band plan
 * (ps_plan_band) to build and apply the masked-band correction of the CG
 * preconditioner.  ps_plan_band makes a plan over the nrings_north rings
 * nearest the equator in each hemisphere (R = 2 nrings_north - 1 rings, the
 * equator ring once), sharing the parent's tables: it must not outlive the
 * parent and runs only the ps_legendre_* calls (ps_synthesis / ps_adjoint
 * return PS_ERR_UNSUPPORTED on it). */
int ps_plan_band(const ps_plan* full, int nrings_north, ps_plan** band);
int ps_legendre_workspace_bytes(const ps_plan* plan, int batch, int spin, int adjoint, size_t* bytes);
int ps_legendre_synthesis(const ps_plan* plan, const double* alm, double* phase, int batch, int spin,
                          void* workspace, size_t workspace_bytes, cudaStream_t stream);
int ps_legendre_adjoint(const ps_plan* plan, const double* phase, double* alm, int batch, int spin, double scale,
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

/* Mixed-size submission (no counterpart in the reference, which calls ducc0 once
 * per map): n single-map transforms of any plans, spins and directions run as one
 * batched ps_synthesis / ps_adjoint per group of equal (plan, direction, spin,
 * scale), largest groups first, in one stream order.  An item's input and output
 * are one map's alm [ncomp][nalm] complex128 or map [ncomp][npix] float64 (ncomp
 * 1 for spin 0, 2 for spin s).  A group whose inputs (outputs) already sit back
 * to back in item order is read (written) in place; otherwise they are gathered
 * into (scattered from) the workspace with one device copy per item.  Nothing is
 * allocated and nothing synchronises, so a submission can be captured in a CUDA
 * graph.  Items must not overlap each other's outputs. */
enum { PS_DIR_SYNTHESIS = 0, PS_DIR_ADJOINT = 1 };
typedef struct ps_work_item {
  const ps_plan* plan;
  int direction; /* PS_DIR_SYNTHESIS: alm -> map; PS_DIR_ADJOINT: map -> alm times scale */
  int spin;
  const double* in;
  double* out;
  double scale; /* adjoint only */
} ps_work_item;
int ps_batch_workspace_bytes(const ps_work_item* items, int n, size_t* bytes);
int ps_batch_submit(const ps_work_item* items, int n, void* workspace, size_t workspace_bytes,
                    cudaStream_t stream);

/* ---------------------------------------------------- pixel-space products
 * Elementwise products of maps of n elements (real = float64, complex =
 * complex128, all contiguous), the per-element products of the reference's
 * Cython kernels, which take [N_r, Npix] arrays and return fresh ones:
 *   op                          inputs (in order)              out   reference
 *   PS_PIX_MULTIPLY             R1 R2 R3                       R     tauNL_utils.pyx:103-113
 *   PS_PIX_MULTIPLY_ASYM        R1A R1B R3A R3B                R     tauNL_utils.pyx:116-126
 *   PS_PIX_MULTIPLYC            R1 R2 C3                       C     tauNL_utils.pyx:129-139
 *   PS_PIX_MULTIPLYC_ASYM       R1A R1B C3A C3B                C     tauNL_utils.pyx:142-152
 *   PS_PIX_MULTIPLYCC           R1 R2 C3                       R     tauNL_utils.pyx:155-165
 *   PS_PIX_MULTIPLYCC_ASYM      R1A R1B R2A R2B C3A C3B        R     tauNL_utils.pyx:168-178
 *   PS_PIX_MULTIPLY2            B1 B2 C1 C2                    R     tauNL_utils.pyx:181-191
 *   PS_PIX_MULTIPLY2R           A B                            R     tauNL_utils.pyx:194-204
 *   PS_PIX_MULTIPLY2C           Ac B                           C     tauNL_utils.pyx:207-217
 *   PS_PIX_MULTIPLYRC           R C                            C     ideal_fisher.pyx:52-60
 *   PS_PIX_MULTIPLYRCSTAR       R C          (fac)             C     ideal_fisher.pyx:64-72
 *   PS_PIX_MULTIPLYRC_SYM       R C R2 C2                      C     ideal_fisher.pyx:76-84
 *   PS_PIX_MULTIPLYRCSTAR_SYM   R C R2 C2    (fac)             C     ideal_fisher.pyx:88-96
 *   PS_PIX_MULTIPLYRR           R1 R2                          R     ideal_fisher.pyx:100-108
 *   PS_PIX_MULTIPLYRR_SYM       R1 R2 R1b R2b                  R     ideal_fisher.pyx:112-120
 *   PS_PIX_R2C / PS_PIX_R2CSTAR re im                          C     ideal_fisher.pyx:18-38
 *   PS_PIX_LENS_PHI             U V ([npol][n] complex each)   C[n]  ideal_fisher.pyx:124-139
 *   PS_PIX_LENS_PHI_SYM         U1 U2 V1 V2                    C[n]  ideal_fisher.pyx:142-157
 *   PS_PIX_PRODUCT_REAL1        A B          (fac)             R     ideal_fisher.pyx:177-190, :325-338
 *   PS_PIX_PRODUCT_REAL2        A0 B0 A1 B1  (fac)             R     the same, two terms of equal weight
 * npol is 1 or 3 for the lensing sums and 1 otherwise; fac is used by the
 * *STAR and PRODUCT_REAL products (the latter are compute_productP_real_all /
 * compute_productQ_real_all for real F maps).  The reference's nthreads argument has no counterpart. */
enum {
  PS_PIX_MULTIPLY = 0, PS_PIX_MULTIPLY_ASYM, PS_PIX_MULTIPLYC, PS_PIX_MULTIPLYC_ASYM, PS_PIX_MULTIPLYCC,
  PS_PIX_MULTIPLYCC_ASYM, PS_PIX_MULTIPLY2, PS_PIX_MULTIPLY2R, PS_PIX_MULTIPLY2C, PS_PIX_MULTIPLYRC,
  PS_PIX_MULTIPLYRCSTAR, PS_PIX_MULTIPLYRC_SYM, PS_PIX_MULTIPLYRCSTAR_SYM, PS_PIX_MULTIPLYRR,
  PS_PIX_MULTIPLYRR_SYM, PS_PIX_R2C, PS_PIX_R2CSTAR, PS_PIX_LENS_PHI, PS_PIX_LENS_PHI_SYM,
  PS_PIX_PRODUCT_REAL1, PS_PIX_PRODUCT_REAL2, PS_PIX_NOPS
};
int ps_pix_product(int op, const void* const* inputs, int n_inputs, void* out, int64_t n, int npol, double fac,
                   cudaStream_t stream);

/* Radial pixel sums  *out = Sum_r w_r tau_r^k Sum_pix f(maps[r][pix])  over maps
 * [nr][npix] (tauNL_utils.pyx:260-405; device scalar out).  tau is read by the
 * DOTDOT (k = 4) and DOTDEL (k = 2) kinds only.  Partial sums are added in a
 * fixed order, so repeated calls give identical results.
 *   PS_SUM_GNL_LOC          P Q                      P^3 Q
 *   PS_SUM_GNL_LOC_DISC     P1 P2 Q1 Q2              P1^2 P2 Q2 + P2^2 P1 Q1
 *   PS_SUM_GNL_CON          R                        R^4
 *   PS_SUM_GNL_CON_DISC     R1 R2                    R1^2 R2^2
 *   PS_SUM_GNL_DOTDOT       A                        tau^4 A^4
 *   PS_SUM_GNL_DOTDOT_DISC  A1 A2                    tau^4 A1^2 A2^2
 *   PS_SUM_GNL_DOTDEL       A B C(complex)           tau^2 A^2 (B^2 + |C|^2)
 *   PS_SUM_GNL_DOTDEL_DISC  A1 A2 B1 B2 C1 C2        tau^2 A1 A2 (B1 B2 + Re C1 C2*)
 *   PS_SUM_GNL_DELDEL       B C                      (B^2 + |C|^2)^2
 *   PS_SUM_GNL_DELDEL_DISC  B1 B2 B3 B4 C1 C2 C3 C4  (B1 B2 + Re C1 C2*)(B3 B4 + Re C3 C4*) */
enum {
  PS_SUM_GNL_LOC = 0, PS_SUM_GNL_LOC_DISC, PS_SUM_GNL_CON, PS_SUM_GNL_CON_DISC, PS_SUM_GNL_DOTDOT,
  PS_SUM_GNL_DOTDOT_DISC, PS_SUM_GNL_DOTDEL, PS_SUM_GNL_DOTDEL_DISC, PS_SUM_GNL_DELDEL, PS_SUM_GNL_DELDEL_DISC,
  PS_SUM_NKINDS
};
int ps_pix_radial_sum_workspace_bytes(int nr, int64_t npix, size_t* bytes);
int ps_pix_radial_sum(int kind, const double* r_weights, const double* tau, const void* const* maps, int n_maps,
                      int nr, int64_t npix, double* out, void* workspace, size_t workspace_bytes,
                      cudaStream_t stream);

/* out[r][lm] = weight Sum_X flX[l][X][r] h_lm[X][lm], l = ls[lm]  (complex128 h_lm
 * [npol][nlm], out [nr][nlm]; npol 1, 2 or 3 -- as in the reference only X = T (npol 1)
 * or X = T, E (npol 2, 3) enter the sum; tauNL_utils.pyx:80-98).  flX is
 * [lsize][npol][nr]; an lm whose l lies outside [0, lsize) gets zeros. */
int ps_apply_fl_weights(const double* flX, int lsize, int npol, int nr, const double* h_lm, const int* ls,
                        int64_t nlm, double weight, double* out, cudaStream_t stream);
/* out[X][lm] = Sum_r lm_map[r][lm] flXs[l][X][r] w_r (tauNL_utils.pyx:220-237); with
 * spin1 != 0, lm_map is [2][nr][nlm] and the sum runs over (lm_map[0] - lm_map[1]) / 2
 * (radial_sum_spin1, tauNL_utils.pyx:240-255).  Complex128 lm_map and out. */
int ps_radial_sum_lm(const double* lm_map, int spin1, const double* r_weights, const double* flXs, int lsize,
                     int npol, int nr, const int* ls, int64_t nlm, double* out, cudaStream_t stream);

/* Fisher outer product of two Q4 arrays, complex128 [4][na][nin] and [4][nb][nin]:
 * fish[a][b] = Re Sum_j (Qa0* Qb0 + Qa1* Qb1 + 9 (Qa2* Qb2 + Qa3* Qb3)
 *                        - 3 (Qa0* Qb3 + Qa1* Qb2 + Qa3* Qb0 + Qa2* Qb1)) / (24 * 48)
 * (outer_product, ideal_fisher.pyx:423-460; sym: square, upper triangle mirrored). */
int ps_outer_product_workspace_bytes(int na, int nb, int64_t nin, size_t* bytes);
int ps_outer_product(const double* Qa, const double* Qb, int na, int nb, int64_t nin, int sym, double* fish,
                     void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------- learned band preconditioner (CG)
 * No counterpart in the reference (its CG offers 'harmonic' and
 * 'pseudo_inverse', polyspec/weighting.py:301-324).  M r = Sigma r +
 * S^1/2 (L_b L_b^T + d_b I) S^1/2 r on band blocks b = (m, 16 consecutive l,
 * fields T, E, B); S = diag(Sigma) (float64 [3][3][nalm]); the network output per
 * block, [48*4 + 1] float32 (L_b row-major, then q_b with d_b = 0.5 tanh q_b), comes
 * from a 3-layer MLP (bf16 weights, FP32 accumulation) trained on (residual,
 * error) pairs of the plain CG.  Blocks are described by the alm
 * index of their first (l, m) and their number of valid l.
 * ps_lbp_moments accumulates C += Sum w u u^T, G += Sum w sym(u t^T), T += Sum
 * w t^T t per block over the real and imaginary parts of `batch` pairs
 * (u = S^1/2 r, t = S^-1/2 (e - Sigma r); r, e complex128 [batch][3][nalm]).
 * ps_lbp_loss_grad gives the per-block loss || (L L^T + d I) u - t ||^2 summed
 * over the pairs (from C, G, T), its gradient with respect to the block's
 * outputs (times scale) and the total loss (fixed order, device double).
 * ps_lbp_apply adds the correction to z. */
int ps_lbp_dims(int* band_l, int* block_dim, int* rank, int* outputs);
int ps_lbp_moments(const int64_t* blk_idx0, const int* blk_nl, int nb, const double* r, const double* e,
                   const double* w, const double* sigma, int batch, int64_t nalm, float* C, float* G, float* T,
                   cudaStream_t stream);
int ps_lbp_loss_grad(const float* L, const float* C, const float* G, const float* T, int nb, float scale, float* dL,
                     float* loss_blk, double* loss, cudaStream_t stream);
int ps_lbp_apply(const int64_t* blk_idx0, const int* blk_nl, int nb, const float* L, const double* sigma,
                 const double* r, double* z, int batch, int64_t nalm, cudaStream_t stream);
/* Dense layer Y[n][o] = act(Sum_i X[n][i] W[o][i] + b[o]) with bf16 W, b and
 * FP32 X, Y, accumulation (in_dim <= 64, out_dim <= 196; act = ReLU or none),
 * its backward pass (dY is overwritten by dY * act'(Y); dX may be null; dW, db
 * reduced over rows in a fixed order) and an Adam step on FP32 master weights
 * that refreshes their bf16 copy. */
int ps_mlp_dense_forward(const float* X, const void* W_bf16, const void* b_bf16, int n, int in_dim, int out_dim,
                         int relu, float* Y, cudaStream_t stream);
int ps_mlp_dense_backward_workspace_bytes(int n, int in_dim, int out_dim, size_t* bytes);
int ps_mlp_dense_backward(float* dY, const float* Y, const float* X, const void* W_bf16, int n, int in_dim,
                          int out_dim, int relu, float* dX, float* dW, float* db, void* workspace,
                          size_t workspace_bytes, cudaStream_t stream);
int ps_mlp_adam(float* param, const float* grad, float* m, float* v, void* param_bf16, int n, float lr, float beta1,
                float beta2, float eps, int step, cudaStream_t stream);

/* ---------------------------------------------- CG vector kernels (harmonic)
 * y[n][a][i] = post[a][i] Sum_b S[a][b][i] pre[b][i] x[n][b][i]: per-(l, m) real 3x3
 * matrices S [3][3][nalm] float64 (Sigma, weighting.py:76-78; C^-1, :60-68) on
 * complex128 vectors [batch][3][nalm]; pre / post [3][nalm] float64 or null (the
 * beam).  ps_lm_dot: out[n] = Sum w[i] Re(x[n][a][i] conj(y[n][a][i])) with w the
 * m weights [nalm] (the CG inner product, weighting.py:255), fixed-order sums. */
int ps_lm_matvec3(const double* S, const double* pre, const double* post, const double* x, double* y, int batch,
                  int64_t nalm, cudaStream_t stream);
int ps_lm_dot_workspace_bytes(int batch, int64_t nalm, size_t* bytes);
int ps_lm_dot(const double* x, const double* y, const double* w, int batch, int64_t nalm, double* out,
              void* workspace, size_t workspace_bytes, cudaStream_t stream);
/* The fused updates of one batched CG step (weighting.py:326-339 per system):
 * ps_lm_matvec3_add: y += S x (the C^-1 term added to the round trip's output);
 * ps_lm_quad_dot: out[n] = Sum w Re(x conj(S x)) without storing S x (the stopping
 * statistic r^T Sigma r; workspace as ps_lm_dot_workspace_bytes);
 * ps_cg_xr_update: x[slot[n]] += alpha[n] p[n], r[n] -= alpha[n] q[n] on rows of `per`
 * complex128 values (slot: int64 [batch] or NULL for the identity: x stays full-size
 * while p, r, q hold the systems still running);
 * ps_cg_direction: p[n] = z[n] + beta[n] p[n]. */
int ps_lm_matvec3_add(const double* S, const double* x, double* y, int batch, int64_t nalm, cudaStream_t stream);
int ps_lm_quad_dot(const double* S, const double* x, const double* w, int batch, int64_t nalm, double* out,
                   void* workspace, size_t workspace_bytes, cudaStream_t stream);
int ps_cg_xr_update(double* x, const int64_t* slot, const double* alpha, const double* p, double* r, const double* q,
                    int batch, int64_t per, cudaStream_t stream);
int ps_cg_direction(double* p, const double* z, const double* beta, int batch, int64_t per, cudaStream_t stream);

/* ------------------------------------------------ masked-band CG preconditioner
 * M r = Sigma r + Sigma B L^H Om^1/2 K_m^-1 Om^1/2 L B Sigma r (per order m; the m = 0 part
 * of the correction real), L the Legendre synthesis stage on a band plan (ps_plan_band) of
 * `plan`, on n = 3 R_b band coordinates (T rings, then Q rings, then U rings).  No
 * counterpart in the reference (its CG offers 'harmonic' and 'pseudo_inverse',
 * polyspec/weighting.py:301-324); built on its weighting (Sigma, :76-78) and CG operator
 * (:297-299).  ps_cutprec_create converts kinv = K_m^-1 (complex64 [mmax+1][n][n]) into the
 * tensor-core layout of the per-m GEMM, BF16 (planes = 1) or BF16 hi + lo (planes = 2), in
 * memory the object owns (enqueued on `stream`); om_half [n], sigma [3][3][nalm] and beam
 * [3][nalm] (float64) stay the caller's.  The band plan must be mixed with the Legendre
 * tables of spins 0 and 2 built on its parent (PS_ERR_UNSUPPORTED otherwise).
 * ps_cutprec_apply: out = M r for r [batch][3][nalm] complex128 (out != r). */
typedef struct ps_cutprec ps_cutprec;
int ps_cutprec_create(const ps_plan* plan, const ps_plan* band, const void* kinv, int n, int planes,
                      const double* om_half, const double* sigma, const double* beam, cudaStream_t stream,
                      ps_cutprec** out);
int ps_cutprec_destroy(ps_cutprec* c);
int ps_cutprec_workspace_bytes(const ps_cutprec* c, int batch, size_t* bytes);
int ps_cutprec_apply(const ps_cutprec* c, const double* r, double* out, int batch, void* workspace,
                     size_t workspace_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------- masked CG solve
 * The conjugate-gradient solve of the optimal S^-1 filter, A x = b with
 *   A = C^-1 + B Y^H W Y B   (CGD._apply_A, polyspec/weighting.py:297-299)
 * and the harmonic preconditioner M = Sigma (weighting.py:306-307), run as the
 * reference's CGD.run(nstep = max_iter, thresh = tol) (weighting.py:217-367) on
 * `batch` independent right-hand sides.  Every system keeps its own alpha, beta
 * and stopping test err = r^T M r / b^T M b (m-weighted inner products,
 * weighting.py:255) and stops at the first step with err < tol, or after
 * max_iter steps; the systems still running are compacted after each step, so
 * the work is the sum of the separate solves' work.
 *
 * ps_cg_create binds a plan and the operator's arrays, all device memory that
 * the caller owns and keeps alive for the object's lifetime:
 *   nfield  1 (T; spin 0) or 3 (T, E, B; spin 0 and spin 2)
 *   inv_cl  C^-1 [nfield][nfield][nalm] float64 (real, per lm)
 *   sigma   Sigma [nfield][nfield][nalm] float64 (the preconditioner)
 *   beam    [nfield][nalm] float64, or NULL (no beam)
 *   weight  the pixel weight W N^-1 W / A_pix, [nfield][npix] float64 (T; T, Q, U)
 *   scale   the adjoint's normalisation (pi / (3 nside^2) for to_lm)
 * The operator runs fused (ps_sht_weighted_roundtrip) on a mixed plan holding
 * the Legendre tables of its spins, else as ps_synthesis, weighting, ps_adjoint.
 *
 * ps_cg_solve: b [batch][nfield][nalm] complex128 (CGD's b0 = B Y^H W N^-1 d);
 * x0 the initial guess in the same layout or NULL (zero); x receives x0 + the
 * CG solution (CGD.get_wiener_lm).  iters [batch] and final_err [batch] are HOST
 * arrays (may be NULL) that receive each system's step count and last err.
 * The call synchronises `stream` once per step to read the stopping tests.  It
 * returns PS_ERR_NOT_CONVERGED, with x holding the last iterate, when a system
 * did not reach tol in max_iter steps (the reference prints a warning then).
 * A system with b^T M b = 0 stops at step 0 with x = x0 and err 0 (the
 * reference divides by zero there). */
typedef struct ps_cg ps_cg;
int ps_cg_create(const ps_plan* plan, int nfield, const double* inv_cl, const double* sigma, const double* beam,
                 const double* weight, double scale, ps_cg** cg);
int ps_cg_destroy(ps_cg* cg);
int ps_cg_workspace_bytes(const ps_cg* cg, int batch, size_t* bytes);
int ps_cg_solve(ps_cg* cg, const double* b, const double* x0, double* x, int batch, int max_iter, double tol,
                int* iters, double* final_err, void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------- binned bispectrum (BSpecBin)
 * Map sets are planar complex: map m is [2][npix] float64 (real plane, then
 * imaginary plane) at maps + 2 m npix; npix must be even, pointers 16-byte aligned.
 *
 * ps_bispec_triplet_sums: out[o] (complex128) = Sum_pix Sum_{t = term_ptr[o]}^{term_ptr[o+1]-1}
 *   M[terms[3t]] M[terms[3t+1]] M[terms[3t+2]] -- the per-triplet pixel sums of
 *   polyspec/bspec_bin.py:339-364 (_analyze3, cubic term), :383-415 (_analyze1, the
 *   linear term over simulations) and :733-755 (ideal numerator), all triplets in one
 *   launch.  Fixed-order reductions (deterministic).  term_ptr [nout+1] and terms
 *   [nterm][3] are int32 device arrays; indices outside [0, nmap) contribute nothing.
 *   PS_ERR_UNSUPPORTED when a 32-pixel tile of all nmap maps exceeds shared memory
 *   (nmap > 440).
 * ps_bispec_pair_products: out[k] (planar [2][npix]) = Sum_{t = ptr[k]}^{ptr[k+1]-1}
 *   s_t op_t(A[a_t]) B[b_t], prods[t] = {a_t, b_t, flags_t}: flags bit 0 conjugates A,
 *   bit 1 negates the term, bits 2-7 hold its multiplicity (0 meaning 1) -- the
 *   products of H maps whose spin-2 and spin-1 adjoint transforms make up
 *   compute_fisher_contribution's Q3 maps (bspec_bin.py:496-518; there as
 *   to_lm_spin(P, M) with M = conj(P), whose real-map inputs are (Re P, Im P)) and
 *   the trispectrum's A and (H A) fields (tspec_bin.py:244-277, 685-730).
 *   nout <= 65535.
 * ps_bispec_assemble_q: out[r][u][lm] (complex128 [nrow][nfield][nlm]) =
 *   scale[u][lm] Sum_c coef[c] V_c(lm) over the contributions c of row r
 *   (row_ptr [nrow+1]; contrib [n][4] int32 = pair, field, l-bin, which) whose field
 *   is u and with edges[bin] <= l_of_lm[lm] < edges[bin+1]; V = conj(G1) - conj(G2)
 *   (which 0) or conj(C1) + conj(C2) (which 1), where A2, A1 [npair][2][nlm]
 *   complex128 hold the (G, C) outputs of the pair's spin-2 and spin-1 adjoints.
 *   The Q3 rows of bspec_bin.py:520-547 (both parities), times the m weights
 *   (S^-1 weighting, :554) or the beam (input of the A^-1 branch, :552).  scale may
 *   be NULL (1); A2 may be NULL (V = conj(G1) or conj(C1): the Q4 rows of
 *   tspec_bin.py:732-773); nrow <= 65535. */
int ps_bispec_triplet_sums_workspace_bytes(int nmap, int64_t npix, int nout, size_t* bytes);
int ps_bispec_triplet_sums(const double* maps, int nmap, int64_t npix, const int* term_ptr, const int* terms,
                           int nout, double* out, void* workspace, size_t workspace_bytes, cudaStream_t stream);
int ps_bispec_pair_products(const double* A, int nA, const double* B, int nB, int64_t npix, const int* ptr,
                            const int* prods, int nout, double* out, cudaStream_t stream);
int ps_bispec_assemble_q(const double* A2, const double* A1, int npair, int64_t nlm, const int* l_of_lm,
                         const int* edges, int nbins, const int* row_ptr, const int* contrib, const double* coef,
                         int nrow, int nfield, const double* scale, double* out, cudaStream_t stream);

/* ------------------------------------------------------------- k-space radial integrals (TSpecTemplate set-up)
 * ps_kint_bessel_table: out[l - lmin][ix] = j_l(x[ix]) for l in [lmin, lmax] (polyspec/cython/
 *   k_integrals.pyx:28-71: x = 0 -> delta_l0; x > 18000 + lmax -> sin(x - l pi/2)/x; zero above the
 *   largest l whose small-x limit exceeds 1e-150).  x [nx] float64 device array.
 * ps_kint_radial: out[l][X][r] += w_l Sum_k (k_i - k_{i-1}) (f_{i-1} + f_i) for l in [lmin, lmax],
 *   X < npol, r < nr, with f_i = kprod[r kstride + i] T[X][l][i] J(k_i r[r]), w_l = (-1)^l (times
 *   sqrt(l(l+1)) if lweight), J = j_{l+nshift} (deriv 0) or (l j_{l-1} - (l+1) j_{l+1})/(2l+1)
 *   (deriv 1), each j linearly interpolated from table (rows tab_lmin .. tab_lmin + tab_nl - 1, on the
 *   grid x, which must start at 0, increase, and reach beyond every k r) -- the q, p, r, a, b and c
 *   integrals of k_integrals.pyx:112-396.  kstride is 0 (one kprod[nk] for all r) or nk (kprod[nr][nk]);
 *   T is [npol][nl_T][nk]; out is [*][npol_out][nr]. */
int ps_kint_bessel_table(const double* x, int64_t nx, int lmin, int lmax, double* out, cudaStream_t stream);
int ps_kint_radial(const double* table, const double* x, int64_t nx, int tab_lmin, int tab_nl, const double* k_arr,
                   int nk, const double* kprod, int kstride, const double* T, int npol, int nl_T,
                   const double* r_arr, int nr, int lmin, int lmax, int nshift, int deriv, int lweight, int npol_out,
                   double* out, cudaStream_t stream);
/* Collider templates (tauNL-light, tauNL-heavy).  Replace compute_collider_F_integral of
 * polyspec/cython/k_integrals.pyx:496-545 (the collider p integral, :399-451, is ps_kint_radial on the real and
 * imaginary parts of its kprod).
 * ps_kint_collider_jlK: jlK[l][k][r] = j_l(K[k] r[r]) linearly interpolated from table [nl][nx] on the grid x
 *   (interpolate_jlkr, :84-110; beyond the grid's end the last interval is extended).
 * ps_kint_collider_F: out [2 nmax_F + 1][nLout][nr][nr] complex: F_{L,L+n}(r_i, r_j) = Sum_k (K_k - K_{k-1})
 *   (f_{k-1} + f_k), f_k = Kprod[k] j_L(K_k r_i) j_{L+n}(K_k r_j) with j from jlK (rows from glmin), for
 *   max(Lmin - nmax_F, 0) <= L <= Lmax + nmax_F, L >= 1, 1 <= L + n <= Lmax + nmax_F; Kprod complex [nK]. */
int ps_kint_collider_jlK(const double* table, const double* x, int64_t nx, int nl, const double* K, int nK,
                         const double* r, int nr, double* jlK, cudaStream_t stream);
int ps_kint_collider_F(const double* jlK, int nl_tab, int glmin, const double* K, int nK, const double* Kprod, int nr,
                       int Lmin, int Lmax, int nmax_F, int nLout, double* out, cudaStream_t stream);
/* ps_tau_sum_collider_diag: tau_sum_n0_collider / tau_sum_nu0_collider (polyspec/cython/tauNL_utils.pyx:877-964):
 *   *out = Sum over rows (rowL, rowM) with Lmin <= L <= Lmax of w_M Re(pref Sum_lam Sum_{j,k} F[L][j][k] w_j w_k
 *   A[lam][row][j] conj(B[lam][row][k])), w_M = 1 (M = 0) or 2; A, B complex [nlam][nrow][nr], F complex
 *   [nLF][nr][nr], nr <= 64.
 * ps_tau_sum_collider_general: tau_sum_general_collider (tauNL_utils.pyx:723-875) for arrays A1 = arr1, A1c = arr1c,
 *   A2 = arr2, A2c = arr2c [2s+1][nrow][nr] (rows of the L-list nLmin..nLmax, m-major), complex F
 *   [2 nmax_F + 1][nLF][nr][nr], coupling coefficients coeffs [s + 1] complex (S = 0, 2, .., 2s); real_beta != 0
 *   doubles the M != 0 rows, otherwise adds the m -> -m piece.  s <= 5, nr <= 64.
 * Workspace of both: ps_tau_collider_workspace_bytes (depends on nrow only). */
int ps_tau_collider_workspace_bytes(int64_t nrow, size_t* bytes);
int ps_tau_sum_collider_diag(const double* A, const double* B, int nlam, const int* rowL, const int* rowM, int nrow,
                             int Lmin, int Lmax, const double* F, int nLF, const double* w, int nr, double pref_re,
                             double pref_im, double* out, void* workspace, size_t workspace_bytes,
                             cudaStream_t stream);
int ps_tau_sum_collider_general(const double* A1, const double* A1c, const double* A2, const double* A2c,
                                const int* rowL, const int* rowM, int nrow, int nLmin, int nLmax, int Lmin, int Lmax,
                                const double* F, int nLF, int nmax_F, const double* w, int nr, int s, int real_beta,
                                const double* coeffs, double* out, void* workspace, size_t workspace_bytes,
                                cudaStream_t stream);
/* ps_convolve_F_collider: convolve_F_general_collider (tauNL_utils.pyx:1197-1355) for one lam1: PQ, cPQ complex
 *   [2s+1][nrow][nr] (the [P^beta Q] and [P^beta* Q] vectors; s = 0: [1][nrow][nr]), complex F [2 nmax_F + 1][nLF][nrF]
 *   [nrF] read at the radial indices inds [nr], S_weights [s + 1] complex (C_S e^{i omega'}, S = 0, 2, .., 2s);
 *   out_re / out_im complex [len(l <= nLmax)][nr] += plus + minus / plus - minus at full_of_row[row].
 * ps_pF_map_complex: compute_pF_map_complex (tauNL_utils.pyx:1357-1446): out complex [npol][nl] += the Gaunt-weighted
 *   shifts of plus / minus (complex [nlm(lmax_in)][nin]) times the complex p [nshift][lsize][npol][nrp] (read at
 *   inds [nin]) and w [nin], for the l-list (ls, ms) and -n1 <= mu1 <= n1. */
int ps_convolve_F_collider(const double* PQ, const double* cPQ, const int* rowL, const int* rowM,
                           const int* full_of_row, int nrow, int nLmin, int nLmax, int Lmin, int Lmax, const double* F,
                           int nLF, int nrF, int nmax_F, const double* w, const int* inds, int nr, int s, int lam1,
                           const double* S_weights, double* out_re, double* out_im, cudaStream_t stream);
int ps_pF_map_complex(const double* plus, const double* minus, int lmax_in, int nin, const double* p, int nshift,
                      int lsize, int npol, int nrp, const double* w, const int* inds, const int* ls, const int* ms,
                      int64_t nl, int n1, int mu1, int nmax, double* out, cudaStream_t stream);

/* ------------------------------------------------------------- ideal bispectrum Fisher (BSpecBin.compute_fisher_ideal)
 * The 3j-symbol sums of polyspec/bspec_bin.py:699-827 as Gauss-Legendre quadratures of binned Wigner d-sums
 * (the Gaunt identity Int d d d dx = 2 (3j)(3j)); no reference counterpart for the individual calls.
 * ps_gl_nodes: n Gauss-Legendre nodes x and weights w on [-1, 1] (device arrays).
 * ps_wigner_binned: Phi[g][b][q][par][k] = Sum_{l in [edges[b], edges[b+1])} H[g][l] s_par(l) d^l_{m_q n_q}(x[k])
 *   for q = 0..3 <-> (m, n) = (-1,-1), (-1,2), (2,-1), (2,2), s_0 = 1, s_1 = (-1)^l; H [G][lmax+1], edges
 *   [nbins+1] ascending with edges[nbins] = lmax + 1 (device arrays).
 * ps_bispec_ideal_contract: out[t][par] = (1/18) Sum_k w[k] Sum_{X,Y} Prod_i Phi[g_i][b_i][(X_i, Y_i)][par][k] over
 *   the m-vectors X, Y in {(-1,-1,2), (2,-1,-1), (-1,2,-1)}, for tasks[t] = (g0, b0, g1, b1, g2, b2) (int32
 *   [ntask][6]); a task with an index out of range gets NaN. */
int ps_gl_nodes(int n, double* x, double* w, cudaStream_t stream);
int ps_wigner_binned(const double* x, int nk, int lmax, const int* edges, int nbins, const double* H, int G,
                     double* Phi, cudaStream_t stream);
int ps_bispec_ideal_contract(const double* Phi, const double* w, int nk, int G, int nbins, const int* tasks, int ntask,
                             double* out, cudaStream_t stream);
/* ps_quad_triple: out[t] = Sum_k w[k] A[ia][k] B[ib][k] C[ic][k] for tasks[t] = (ia, ib, ic) (int32 [ntask][3];
 *   A [nA][nk], B [nB][nk], C [nC][nk]); an index out of range gives NaN.  Used with ps_wigner_binned rows for
 *   the (l1 l2 L; -1 -1 2)^2 sums of TSpecBin's ideal 0- and 2-field terms (polyspec/tspec_bin.py:883-1045). */
int ps_quad_triple(const double* A, int nA, const double* B, int nB, const double* C, int nC, const double* w, int nk,
                   const int* tasks, int ntask, double* out, cudaStream_t stream);

/* ------------------------------------------------------------- small-momentum 3j / Gaunt coefficients
 * ps_gaunt_table: out[i] = (l1 l2 n; m1 m2 m3) (gaunt = 0) or the Gaunt coefficient
 *   sqrt((2l1+1)(2l2+1)(2n+1)/4pi) (l1 l2 n; 0 0 0)(l1 l2 n; m1 m2 m3) (gaunt = 1, the gaunt_symbol of
 *   polyspec/cython/tauNL_utils.pyx:1716-1718) for args[i] = (l1, l2, n, m1, m2, m3) (int32 [n][6], device),
 *   n a small momentum (the direction-dependent tauNL orders); evaluation by short-product Racah sums. */
int ps_gaunt_table(const int* args, int n, int gaunt, double* out, cudaStream_t stream);
/* ps_shift_weight_map_all: the Gaunt-weighted l-shifts of polyspec/cython/tauNL_utils.pyx:407-512 as a
 *   gather.  flX [nshift = 2 nmax + 1][lsize][npol][nr] (the p_{l,l+n}^X(r) integrals), h [npol][nsrc] complex
 *   harmonics of the source lm list (l = src_l[s]; src_of_lm maps the m-major index of l, m <= lmax_src to a
 *   source or -1), targets (tL, tK) the m-major list of l <= lmax_src + n; Lre, Lim complex [nr][ntarget] are
 *   accumulated in place; weight complex; 0 <= mu <= n <= nmax.  Workspace: ps_shift_weight_workspace_bytes. */
/* ps_pF_map_real: out[u][i] (complex [npol][nl]) += the Gaunt-weighted gather of compute_pF_map_real
 *   (polyspec/cython/tauNL_utils.pyx:1531-1620): inputs plus/minus complex [nlm(lmax_in)][nin], p the p_lL^X
 *   integrals [nshift = 2 nmax + 1][lsize][npol][nrp], radial weights w [nin] and sample indices inds [nin],
 *   sources (ls, ms) [nl].
 * ps_product_pnmu_sym: out[t] = Sum_k w_k [Re(P[pq_k][0][t] F[f_k][0][t]) + 2 Sum_{mu=1..n1} Re(P[pq_k][mu][t]
 *   F[f_k][mu][t])] (compute_productPnmu_sym_all, polyspec/cython/ideal_fisher.pyx:195-212), complex P, F.
 * ps_product_q_complex: out[t] = Sum_k w_k Q[pq_k][t] F[f_k][mu1][t] (compute_productQ_complex_all,
 *   ideal_fisher.pyx:343-357), real Q, complex F [nF][nmu][ntot], complex out. */
int ps_pF_map_real(const double* plus, const double* minus, int lmax_in, int nin, const double* p, int nshift, int lsize,
                   int npol, int nrp, const double* w, const int* inds, const int* ls, const int* ms, int64_t nl, int n1,
                   int mu1, int nmax, double* out, cudaStream_t stream);
int ps_product_pnmu_sym(const double* P, const double* F, int n1, int64_t ntot, const double* wts, const int* pq,
                        const int* fi, int nw, double* out, cudaStream_t stream);
int ps_product_q_complex(const double* Q, const double* F, int nmu, int mu1, int64_t ntot, const double* wts,
                         const int* pq, const int* fi, int nw, double* out, cudaStream_t stream);
/* ps_tau_sum_general: *out = tau_sum_general of polyspec/cython/tauNL_utils.pyx:650-715 for A [2n1+1][nrow][nr],
 *   B [2n3+1][nrow][nr] (complex, rows (rowL, rowM) of the L-list, row_of_full mapping the m-major index of (L, |M|),
 *   L <= nLmax, to a row or -1), FT [2 nmax_F + 1][nLF][nr][nr] = the reference's FLLs with its two radial axes
 *   swapped (FT[..][k][j] = F_{L,L+Delta}(r_j, r'_k)), radial weights w [nr].  Workspace:
 *   ps_tau_general_workspace_bytes.
 * ps_convolve_F_general: convolve_F_general of tauNL_utils.pyx:1069-1180 for one mu1: out_re/out_im complex
 *   [len(l <= nLmax)][nr] += plus +- minus at full_of_row[row] for rows with Lmin <= L <= Lmax; PQ [2n3+1][nrow][nr],
 *   FT [2 nmax_F + 1][nLF][nrF][nrF] (radial axes swapped as above) read at the radial indices inds [nr]. */
/* ps_gaunt_row_table: gtab [nrow][n + 1][2n + 1][2], the Gaunt coefficients of every row for Delta = -n, -n+2, .., n,
 *   mu = -n..n: part 0 Gaunt(L, L+Delta, n; -M, M-mu, mu), part 1 Gaunt(L, L+Delta, n; M, -M-mu, mu) (0 outside
 *   Lmin <= L, L+Delta <= Lmax or |M'| > L+Delta); computed once per n and passed to the two contractions.
 *   The gtab given to ps_tau_sum_general / ps_convolve_F_general must come from this function called with the
 *   same (rowL, rowM, nrow, Lmin, Lmax, n) as the contraction: nothing checks this, and a table built for other
 *   rows or another L range silently drops or keeps the wrong coupling terms.  The workspace of
 *   ps_tau_sum_general depends on the current device's SM count: query it on the device that runs the call. */
int ps_gaunt_row_table(const int* rowL, const int* rowM, int nrow, int Lmin, int Lmax, int n, double* gtab,
                       cudaStream_t stream);
int ps_tau_general_workspace_bytes(int nrow, int nr, size_t* bytes);
int ps_tau_sum_general(const double* A, const double* B, const int* row_of_full, const int* rowL, const int* rowM,
                       int nrow, int nLmax, int Lmin, int Lmax, const double* F, int nLF, int nmax_F, const double* w,
                       int nr, int n1, int n3, int n, const double* gtab, double* out, void* workspace,
                       size_t workspace_bytes, cudaStream_t stream);
int ps_convolve_F_general(const double* PQ, const int* row_of_full, const int* rowL, const int* rowM,
                          const int* full_of_row, int nrow, int nLmax, int Lmin, int Lmax, const double* F, int nLF,
                          int nrF, int nmax_F, const double* w, const int* inds, int nr, int n1, int n3, int n, int mu1,
                          const double* gtab, double* out_re, double* out_im, cudaStream_t stream);
int ps_shift_weight_workspace_bytes(int64_t ntarget, int n, size_t* bytes);
int ps_shift_weight_map_all(const double* flX, int nshift, int lsize, int npol, int nr, const double* h, int64_t nsrc,
                            const int* src_l, const int* src_of_lm, int lmax_src, const int* tL, const int* tK,
                            int64_t ntarget, int n, int mu, double weight_re, double weight_im, int nmax, double* Lre,
                            double* Lim, void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* ------------------------------------------------------------- inpainting (Weightings.inpaint_map)
 * ps_healpix_neighbours: out[p][k] (int32 [12 nside^2][8]) = the RING neighbours of pixel p in the order
 *   SW, W, NW, N, NE, E, SE, S, -1 where there are only 7 -- healpy.get_all_neighbours, which
 *   polyspec/weighting.py:118, :138 calls.  tables (device int32 [2][9][12]): per 3 x 3 cell (cx + 3 cy,
 *   cx/cy 0 below, 1 inside, 2 above the face's lattice) and face, the adjacent face (-1: none) and the
 *   lattice symmetry bits (1 flip x, 2 flip y, 4 swap), as polyspec_b200/healpix.py derives them.
 * ps_inpaint_average: dst[pix[i]] = the average of src over the 8 neighbours of pix[i] (nb from
 *   ps_healpix_neighbours; -1 reads src[npix - 1]): the plain mean (weighted = 0, the smoothing passes of
 *   weighting.py:135-141) or the mean weighted by (value != 1e-30) (weighted = 1, the fill passes of
 *   :115-131).  dst must not alias src; entries of dst outside the list are left as they are. */
int ps_healpix_neighbours(int nside, const int* tables, int* out, cudaStream_t stream);
int ps_inpaint_average(const double* src, const int* pix, int64_t n, const int* nb, int64_t npix, int weighted,
                       double* dst, cudaStream_t stream);

/* ------------------------------------------------------------- local tauNL (TSpecTemplate 'tauNL-loc')
 * ps_tau_F_integral: F[n + nmax_F][L][i][j] = F_{L,L+n}(r_i, r_j) for n in [-nmax_F, nmax_F], the closed
 *   form of polyspec/cython/k_integrals.pyx:453-494 (compute_F_integral; reference pref argument, the
 *   2^(ns-3) factor applied here) for L in [max(Lmin - nmax_F, 0), Lmax + nmax_F] with L, L + n >= 1;
 *   other entries are left as they are.  F has (2 nmax_F + 1) * nL * nr * nr doubles, nL >= Lmax +
 *   nmax_F + 1.  *err (device int) is set to 1 where a hypergeometric series did not converge.
 * ps_tau_convolve_F: out[j][lm] = Sum_k F_L(r_j, r_k) w_k X[k][lm] / sqrt(4 pi) with L = lm_L[lm] (-1:
 *   out = 0, else L < nL), the convolve_F_n000 of polyspec/cython/tauNL_utils.pyx:966-995 over a full lm
 *   list; X, out complex [nr][nlm], F one n-slice stored transposed, [nr][nr][nL] (F[j][k][L]).  With dot != NULL (device double) also
 *   *dot = Sum_{lm,j} lm_w[lm] w_j Re(A[j][lm] conj(out[j][lm])) -- tau_sum_n0 of
 *   tauNL_utils.pyx:604-647 for (A, X) -- using a workspace of ps_tau_convolve_workspace_bytes; out
 *   may then be NULL.  nr <= 384. */
int ps_tau_F_integral(const double* r_arr, int nr, int Lmin, int Lmax, int nmax_F, int nL, double ns, double pref,
                      double* F, int* err, cudaStream_t stream);
int ps_tau_convolve_workspace_bytes(int64_t nlm, size_t* bytes);
int ps_tau_convolve_F(const double* X, const double* A, const int* lm_L, const double* lm_w, const double* F, int nL,
                      const double* r_weights, int nr, int64_t nlm, double* out, double* dot, void* workspace,
                      size_t workspace_bytes, cudaStream_t stream);

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
