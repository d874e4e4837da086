/*
 * sinvb.h -- C ABI of libsinvb.so, the B200 (sm_100a) selected-inversion library.
 *
 * Selected inversion of a block-tridiagonal matrix A with n diagonal blocks
 * of size b x b: the diagonal blocks G_ii, the upper blocks G_{i,i+1} and the
 * lower blocks G_{i+1,i} of G = A^{-1}.
 *
 * Block-array layout (the reference's ``convertDenseToBlkTridiag``,
 * src/sinv/utils/matrices_utils.py:115-151): ``diag`` holds n blocks,
 * ``upper`` n-1 blocks A_{i,i+1}, ``lower`` n-1 blocks A_{i+1,i}; every
 * block is b x b, row-major, contiguous, blocks back to back.  Complex
 * element types are interleaved (re, im) pairs (C99 / numpy / torch layout).
 *
 * All pointers are device pointers.  Every call is asynchronous on
 * ``stream``: it validates arguments on the host (negative return codes),
 * enqueues its kernels and returns.  Conditions found on the device (a zero
 * or non-finite pivot in the pivot-free elimination, a wait that gave up)
 * are written to a status word inside the caller's workspace and read back
 * with ``sinvb_workspace_status``.  The library never allocates or frees
 * device memory of its own in these entry points: the caller passes a
 * workspace of at least ``sinvb_*_workspace_size`` bytes.  Inputs are never
 * modified.  Calls on different streams with different workspaces may run
 * concurrently.
 */
#ifndef SINVB_H
#define SINVB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* sinvb_stream_t; /* == cudaStream_t */

/* ---- return / status codes ------------------------------------------- */
#define SINVB_OK 0
#define SINVB_EINVAL (-1)      /* bad argument (null pointer, size, flags)     */
#define SINVB_ECUDA (-2)       /* a CUDA runtime call failed                   */
#define SINVB_EWORKSPACE (-3)  /* workspace too small or misaligned            */
#define SINVB_EUNSUPPORTED (-4)/* no B200 / sm_100 device, or feature missing  */
/* device-detected, reported through the workspace status word (>0) */
#define SINVB_STATUS_PIVOT 1   /* zero or non-finite pivot in a block inverse  */
#define SINVB_STATUS_TIMEOUT 2 /* a bounded device wait gave up                */

/* ---- flags -------------------------------------------------------------- */
/* rgf.py:19 sym_mat: G_{i,i+1} = G_{i+1,i}^T (plain transpose, rgf.py:57-58) */
#define SINVB_SYM 1u
/* rgf.py:20 save_off_diag: write G_upper / G_lower (rgf.py:55) */
#define SINVB_SAVE_OFFDIAG 2u
/* run the sweep with the whole GPU as one team (cooperative launch) even for
 * small blocks; by default the library picks the team from b */
#define SINVB_FORCE_GRID 4u
#define SINVB_FORCE_CTA 8u
/* overwrite the inputs with the results: G_diag -> diag, G_upper -> upper,
 * G_lower -> lower (the G_* arguments are ignored; requires SAVE_OFFDIAG).
 * Halves the memory of a call; the reference never does this (rgf.py:41
 * copies), so the Python layer uses it only when asked. */
#define SINVB_INPLACE 16u

/* ---- element type codes --------------------------------------------------- */
#define SINVB_C128 0 /* complex double */
#define SINVB_F64 1  /* double         */
#define SINVB_C64 2  /* complex float  (computed in FP64, rounded on output) */
#define SINVB_F32 3  /* float          (computed in FP64, rounded on output) */

/* Library / device info. */
int sinvb_version(void);
const char* sinvb_status_string(int code);

/* Bytes of workspace one ``sinvb_rgf_*`` call needs (256-byte aligned). */
size_t sinvb_rgf_workspace_size(int n, int b, int dtype, unsigned flags);

/*
 * Serial RGF selected inversion.
 * Replaces ``rgf(A, sym_mat, save_off_diag)`` of
 * src/sinv/algorithms/rgf/rgf.py:17-64 (forward sweep :44-48, backward sweep
 * :51-62) in the block-array form of
 * src/sinv/algorithms/rgf/rgf2sided.py:18-24.
 * G_upper / G_lower may be NULL when SINVB_SAVE_OFFDIAG is not set.
 */
int sinvb_rgf_z(const void* diag, const void* upper, const void* lower, int n, int b,
                unsigned flags, void* G_diag, void* G_upper, void* G_lower,
                void* workspace, size_t workspace_bytes, sinvb_stream_t stream);
int sinvb_rgf_d(const void* diag, const void* upper, const void* lower, int n, int b,
                unsigned flags, void* G_diag, void* G_upper, void* G_lower,
                void* workspace, size_t workspace_bytes, sinvb_stream_t stream);
int sinvb_rgf_c(const void* diag, const void* upper, const void* lower, int n, int b,
                unsigned flags, void* G_diag, void* G_upper, void* G_lower,
                void* workspace, size_t workspace_bytes, sinvb_stream_t stream);
int sinvb_rgf_s(const void* diag, const void* upper, const void* lower, int n, int b,
                unsigned flags, void* G_diag, void* G_upper, void* G_lower,
                void* workspace, size_t workspace_bytes, sinvb_stream_t stream);

/*
 * Two-sided RGF on one GPU.  Replaces ``rgf2sided(A_diag, A_upper, A_lower,
 * sym_mat, save_off_diag)`` of src/sinv/algorithms/rgf/rgf2sided.py:18-274
 * (two MPI processes sweeping towards the middle) with two teams of CTAs of
 * one launch: the dependency chain of a single matrix is about n/2 block
 * steps instead of n.  Same arrays and results as sinvb_rgf_*; requires
 * SINVB_SAVE_OFFDIAG (the halves keep their X / P blocks in G_upper and
 * G_lower); SINVB_SYM allowed; complex128 and float64.
 */
size_t sinvb_rgf2s_workspace_size(int n, int b, int dtype, unsigned flags);
int sinvb_rgf2s_z(const void* diag, const void* upper, const void* lower, int n, int b,
                  unsigned flags, void* G_diag, void* G_upper, void* G_lower,
                  void* workspace, size_t workspace_bytes, sinvb_stream_t stream);
int sinvb_rgf2s_d(const void* diag, const void* upper, const void* lower, int n, int b,
                  unsigned flags, void* G_diag, void* G_upper, void* G_lower,
                  void* workspace, size_t workspace_bytes, sinvb_stream_t stream);

/*
 * Device status word of a workspace: synchronises ``stream`` and returns the
 * status (SINVB_OK or a positive SINVB_STATUS_*) in *status.  The word is
 * reset by the next call that uses the workspace.
 */
int sinvb_workspace_status(const void* workspace, sinvb_stream_t stream, int* status);

/* ---- lesser Green's function ------------------------------------------------- */
/*
 * No reference counterpart: the step a transport code takes after rgf
 * (src/sinv/algorithms/rgf/rgf.py:17-64) at each energy, G< = G Sigma< G^H on
 * the tridiagonal blocks for a block-diagonal lesser self-energy
 * (``sigma_lesser``: n blocks).  Writes the retarded blocks as sinvb_rgf_z
 * with SAVE_OFFDIAG, and GL_diag (n blocks G<_ii), GL_upper (n-1 blocks
 * G<_{i,i+1}); G<_{i+1,i} = -(G<_{i,i+1})^H.  complex128; flags: FORCE_CTA or
 * FORCE_GRID only.
 */
size_t sinvb_rgf_lesser_workspace_size(int n, int b);
int sinvb_rgf_lesser_z(const void* diag, const void* upper, const void* lower, const void* sigma_lesser, int n,
                       int b, unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* GL_diag,
                       void* GL_upper, void* workspace, size_t workspace_bytes, sinvb_stream_t stream);

/*
 * Many energies of a transport calculation's loop at once: for every
 * descriptor, the outputs of sinvb_rgf_lesser_z on its own matrix and
 * self-energy (own n and b), all in one persistent launch whose teams of
 * CTAs take whole instances from a device queue (largest b^3 n first).  No
 * reference counterpart: the caller-side loop of rgf
 * (src/sinv/algorithms/rgf/rgf.py:17-64) followed by G Sigma< G^H per energy.
 * complex128; flags: 0 or SINVB_FORCE_CTA (one-CTA teams).  ``status`` (count
 * ints on the device, or NULL) receives each instance's SINVB_OK /
 * SINVB_STATUS_*; the workspace status word holds the first failure.  Outputs
 * must not overlap the inputs.
 */
typedef struct sinvb_lesser_desc {
  const void* diag;
  const void* upper;
  const void* lower;
  const void* sigma_lesser;  /* n blocks */
  void* G_diag;
  void* G_upper;
  void* G_lower;
  void* GL_diag;             /* n blocks G<_ii */
  void* GL_upper;            /* n-1 blocks G<_{i,i+1} */
  int n;
  int b;
} sinvb_lesser_desc;
size_t sinvb_rgf_lesser_batched_workspace_size(const sinvb_lesser_desc* descs, int count, unsigned flags);
int sinvb_rgf_lesser_batched_z(const sinvb_lesser_desc* descs, int count, unsigned flags, void* workspace,
                               size_t workspace_bytes, int* status, sinvb_stream_t stream);

/* ---- adjoint (reverse mode) of the RGF sweeps ------------------------------------ */
/*
 * No reference counterpart (the reference has no gradients); the adjoint of
 * src/sinv/algorithms/rgf/rgf.py:44-62.  The forward call saves checkpoints
 * g_{s*c-1} (c = ceil(sqrt(n)), sinvb_rgf_checkpoints gives c and the count)
 * so the adjoint recomputes the left-connected blocks instead of storing all
 * of them.  Requires SINVB_SAVE_OFFDIAG.  Upstream adjoints bG_* follow the
 * torch convention (dL/dG* for complex, dL/dG for real); bG_upper / bG_lower
 * may be NULL (zero).  Outputs aD (n blocks), aU, aL (n-1 blocks): dL/dA* on
 * the tridiagonal pattern.
 */
int sinvb_rgf_checkpoints(int n, int* every, int* count);
int sinvb_rgf_forward_ckpt_z(const void* diag, const void* upper, const void* lower, int n, int b,
                             unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* checkpoints,
                             int every, void* workspace, size_t workspace_bytes, sinvb_stream_t stream);
int sinvb_rgf_forward_ckpt_d(const void* diag, const void* upper, const void* lower, int n, int b,
                             unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* checkpoints,
                             int every, void* workspace, size_t workspace_bytes, sinvb_stream_t stream);
size_t sinvb_rgf_adjoint_workspace_size(int n, int b, int dtype, unsigned flags);
int sinvb_rgf_adjoint_z(const void* diag, const void* upper, const void* lower, const void* G_diag,
                        const void* G_upper, const void* G_lower, const void* bG_diag, const void* bG_upper,
                        const void* bG_lower, const void* checkpoints, int every, int n, int b, unsigned flags,
                        void* aD, void* aU, void* aL, void* workspace, size_t workspace_bytes,
                        sinvb_stream_t stream);
int sinvb_rgf_adjoint_d(const void* diag, const void* upper, const void* lower, const void* G_diag,
                        const void* G_upper, const void* G_lower, const void* bG_diag, const void* bG_upper,
                        const void* bG_lower, const void* checkpoints, int every, int n, int b, unsigned flags,
                        void* aD, void* aU, void* aL, void* workspace, size_t workspace_bytes,
                        sinvb_stream_t stream);

/* ---- BCR: block cyclic reduction on the whole GPU ------------------------------ */
/*
 * Replaces ``bcr_serial(A, blocksize)`` of
 * src/sinv/algorithms/bcr/bcr_serial.py:19-62 (reduce :66-216, root inverse
 * :220-249, production :253-466; padding and index sets of
 * src/sinv/algorithms/bcr/bcr_utils.py:17-129) in block-array form: the
 * G_ii, G_{i,i+1}, G_{i+1,i} blocks the reference's dense result holds.  The
 * rows of each reduction / production level run in parallel on every SM.
 */
size_t sinvb_bcr_workspace_size(int n, int b, int dtype, unsigned flags);
int sinvb_bcr_z(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream);
int sinvb_bcr_d(const void* diag, const void* upper, const void* lower, int n, int b, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream);

/* ---- batched RGF: many independent matrices in one persistent launch ------- */
/*
 * One matrix of a batch (block arrays as above; every instance may have its
 * own n and b).  This is the energy loop of a transport calculation: the
 * reference calls rgf (src/sinv/algorithms/rgf/rgf.py:17) once per matrix
 * A(E_k) = E_k I - H - Sigma(E_k); here one launch walks every instance's
 * sweep, instances dispatched largest-first from a device work queue, one
 * team of CTAs per instance.
 */
typedef struct sinvb_batch_desc {
  const void* diag;
  const void* upper;
  const void* lower;
  void* G_diag;
  void* G_upper;
  void* G_lower;
  int n;
  int b;
} sinvb_batch_desc;

/* precision modes of the batched call (the ``flags`` argument, high bits) */
#define SINVB_PREC_FP64 0u          /* every product in FP64 (DMMA)             */
#define SINVB_PREC_MIXED (1u << 8)  /* block products on tcgen05, FP64 inverses */
/* int8 slices per value of the mixed products (1..8) in flag bits 12-15; 0 means 7 */
#define SINVB_PREC_DIGITS(d) (((unsigned)(d) & 15u) << 12)

size_t sinvb_rgf_batched_workspace_size(const sinvb_batch_desc* descs, int count, int dtype, unsigned flags);

/*
 * Uploads the descriptors into the workspace (ordered by cost) and launches
 * the persistent kernel.  ``status`` (optional, device, ``count`` ints) gets
 * each instance's device status, indexed like ``descs``.
 */
int sinvb_rgf_batched_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream);
int sinvb_rgf_batched_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream);
/*
 * Streamed form of the batched call, for inputs still arriving from the host:
 * instance k (index into ``descs``) starts only once the device word
 * ``ready[k]`` equals ``gen`` (the caller's copy stream writes it after the
 * instance's inputs, in stream order), and on finishing the kernel sets
 * ``done[k] = gen`` (system scope) so the caller can start copying its
 * results out while the launch runs on.  Waits are bounded (status
 * SINVB_STATUS_TIMEOUT).  ``gen`` must differ from every value the two
 * arrays held before (a call counter); ``ready`` / ``done``: ``count``
 * device words each.  Instances are taken largest b^3 n first, so the caller
 * should copy them in that order.
 */
int sinvb_rgf_batched_stream_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                               size_t workspace_bytes, int* status, const unsigned* ready, unsigned* done,
                               unsigned gen, sinvb_stream_t stream);
int sinvb_rgf_batched_stream_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                               size_t workspace_bytes, int* status, const unsigned* ready, unsigned* done,
                               unsigned gen, sinvb_stream_t stream);
/*
 * Re-runs the batch last uploaded into ``workspace`` (same descriptors, same
 * buffers) with no host-to-device traffic: one memset and one kernel launch,
 * suitable for stream capture into a CUDA graph.
 */
int sinvb_rgf_batched_rerun_z(void* workspace, sinvb_stream_t stream);
int sinvb_rgf_batched_rerun_d(void* workspace, sinvb_stream_t stream);
/*
 * A schedule for the batched call, as the autotuner (sinv_b200/autotune.py)
 * chooses it from measured per-block-row costs; no reference counterpart
 * (the reference inverts one matrix per rgf call, rgf.py:17).  Arrays are
 * indexed like ``descs``; every field may be left 0 / NULL for the
 * library's rule (teams of 1 / 2 / 4 / 8 CTAs for b < 256 / 256 / 512 / 1024,
 * queue ordered by b^3 n, int8 products from b = 256 on).
 */
typedef struct sinvb_batch_schedule {
  const int* team;        /* CTAs of each instance's team (0: the rule), at most the SM count */
  const float* priority;  /* queue order, highest first (NULL: b^3 n) */
  int mixed_min_b;        /* mixed batches: smallest b with int8 products (0: 256) */
  int reserved;
} sinvb_batch_schedule;

size_t sinvb_rgf_batched_sched_workspace_size(const sinvb_batch_desc* descs, int count, int dtype,
                                              unsigned flags, const sinvb_batch_schedule* sched);
/* sinvb_rgf_batched_z / _d with a schedule (NULL: as without). */
int sinvb_rgf_batched_sched_z(const sinvb_batch_desc* descs, int count, unsigned flags,
                              const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes,
                              int* status, sinvb_stream_t stream);
int sinvb_rgf_batched_sched_d(const sinvb_batch_desc* descs, int count, unsigned flags,
                              const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes,
                              int* status, sinvb_stream_t stream);
/* sinvb_rgf_batched_stream_z / _d with a schedule (NULL: as without).  The
 * queue takes the instances in descending priority, ties in descriptor order;
 * the caller copies them in that order. */
int sinvb_rgf_batched_stream_sched_z(const sinvb_batch_desc* descs, int count, unsigned flags,
                                     const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes,
                                     int* status, const unsigned* ready, unsigned* done, unsigned gen,
                                     sinvb_stream_t stream);
int sinvb_rgf_batched_stream_sched_d(const sinvb_batch_desc* descs, int count, unsigned flags,
                                     const sinvb_batch_schedule* sched, void* workspace, size_t workspace_bytes,
                                     int* status, const unsigned* ready, unsigned* done, unsigned gen,
                                     sinvb_stream_t stream);

/*
 * Batched forward sweeps that also save the adjoint's checkpoints (the
 * batched form of sinvb_rgf_forward_ckpt_*; no reference counterpart, the
 * reference has no gradients): instance k writes g_{s*c-1}, c =
 * ceil(sqrt(n_k)), into checkpoints[k], a device array of the count blocks
 * sinvb_rgf_checkpoints(n_k) gives (NULL allowed when that count is 0).
 * FP64 products only, not in place.
 */
int sinvb_rgf_batched_ckpt_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* const* checkpoints,
                             void* workspace, size_t workspace_bytes, int* status, sinvb_stream_t stream);
int sinvb_rgf_batched_ckpt_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* const* checkpoints,
                             void* workspace, size_t workspace_bytes, int* status, sinvb_stream_t stream);

/*
 * Batched adjoint: the reverse of both sweeps (rgf.py:44-62) of many
 * instances in one persistent launch, as sinvb_rgf_adjoint_* for each
 * (checkpoints from sinvb_rgf_batched_ckpt_* or sinvb_rgf_forward_ckpt_*).
 * No reference counterpart.  Per instance: inputs A, the forward results G,
 * upstream adjoints bG (bG_upper / bG_lower may be NULL), checkpoints, and
 * the outputs aD (n blocks), aU, aL (n-1 blocks).  flags: SINVB_SYM,
 * SINVB_SAVE_OFFDIAG, SINVB_FORCE_CTA.  ``status``: per-instance device
 * status (optional).
 */
typedef struct sinvb_adjoint_desc {
  const void* diag;
  const void* upper;
  const void* lower;
  const void* G_diag;
  const void* G_upper;
  const void* G_lower;
  const void* bG_diag;
  const void* bG_upper;
  const void* bG_lower;
  const void* checkpoints;
  void* aD;
  void* aU;
  void* aL;
  int n;
  int b;
} sinvb_adjoint_desc;

size_t sinvb_rgf_adjoint_batched_workspace_size(const sinvb_adjoint_desc* descs, int count, int dtype,
                                                unsigned flags);
int sinvb_rgf_adjoint_batched_z(const sinvb_adjoint_desc* descs, int count, unsigned flags, void* workspace,
                                size_t workspace_bytes, int* status, sinvb_stream_t stream);
int sinvb_rgf_adjoint_batched_d(const sinvb_adjoint_desc* descs, int count, unsigned flags, void* workspace,
                                size_t workspace_bytes, int* status, sinvb_stream_t stream);

/*
 * No reference counterpart (the reference has no device waits; its failure
 * analogue is LinAlgError from rgf.py:44,48).  Bound, in seconds, of every
 * device-side wait of the batched launches that use ``workspace`` from now
 * on: team barriers, scratch slots and streamed ready words (default 60 s).
 * A wait that reaches it reports SINVB_STATUS_TIMEOUT for its instance,
 * which is then abandoned, and the launch goes on with the others.  Host-side
 * setting, kept per workspace address; 0 < seconds <= 3600.
 */
int sinvb_rgf_batched_set_wait_limit(const void* workspace, double seconds);

/* ---- PSR: parallel Schur reduction over partitions of one matrix -------------- */
/*
 * psr_seqsolve (src/sinv/algorithms/psr/psr_seqsolve.py:20-73): the block
 * rows are split into ``partitions`` parts as psr_utils.py:61-100 does (n / P
 * rows each, the remainder in the first); every part is reduced by its own
 * team of CTAs, the 2(P-1) boundary rows form a block tridiagonal reduced
 * system inverted by the whole grid, and every team then produces its part's
 * blocks.  The MPI processes of the reference are the teams of one launch.
 * ``partitions`` = 0 picks about sqrt(n/2); otherwise 3 <= P <= 32 and
 * n >= 3P (psr_utils.py:55-58), else SINVB_EINVAL.  ``flags`` must be 0; the
 * whole tridiagonal part of the inverse is written.
 * sinvb_psr_partitions returns the P a call with these arguments uses, or -1.
 */
int sinvb_psr_partitions(int n, int partitions);
size_t sinvb_psr_workspace_size(int n, int b, int partitions, int dtype, unsigned flags);
int sinvb_psr_z(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream);
int sinvb_psr_d(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, unsigned flags,
                void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                sinvb_stream_t stream);
/*
 * One partition of a multi-GPU PSR on this GPU: what reference process
 * ``part`` of ``partitions`` does (psr_seqsolve.py:52-70), holding only its
 * own block rows t .. B (m = B - t + 1 rows; the partitions are those of
 * psr_utils.py:61-100).  diag: m blocks; upper / lower: the couplings
 * A[i,i+1] / A[i+1,i] of rows t .. B (m blocks, m - 1 for the last partition);
 * G_diag / G_upper / G_lower: the same shapes.  stage 0 reduces the partition
 * and writes six b x b slots to ``boundary`` (device): its part of the
 * reduced system (first partition D[B]; last D[t]; central D[t], D[B],
 * A[t,B], A[B,t]) and in slots 4, 5 the couplings A[B,B+1], A[B+1,B] to the
 * next partition (zero for the last).  stage 1 takes the boundary blocks of
 * the reduced system's inverse in slots 0-3 (G[B,B]; G[t,t]; G[t,t], G[B,B],
 * G[t,B], G[B,t]) and writes the partition's blocks; the couplings to the
 * next partition, G[B,B+1] and G[B+1,B] (element m - 1 of G_upper /
 * G_lower), come from the reduced inverse and are the caller's to store.
 * Use one workspace of sinvb_psr_part_workspace_size bytes for both stages.
 */
size_t sinvb_psr_part_workspace_size(int n, int b, int partitions, int part, int dtype);
int sinvb_psr_part_z(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, int part,
                     int stage, void* boundary, void* G_diag, void* G_upper, void* G_lower, void* workspace,
                     size_t workspace_bytes, sinvb_stream_t stream);
int sinvb_psr_part_d(const void* diag, const void* upper, const void* lower, int n, int b, int partitions, int part,
                     int stage, void* boundary, void* G_diag, void* G_upper, void* G_lower, void* workspace,
                     size_t workspace_bytes, sinvb_stream_t stream);

/* ---- PDIV: pairwise divide and conquer over partitions of one matrix ---------- */
/*
 * pdiv_localmap (src/sinv/algorithms/pdiv/pdiv_localmap.py:27-91) of all
 * ``partitions`` processes at once: the block rows are split as
 * pdiv_utils.py:84-123 does (n / P rows each, the remainder in the first);
 * every partition's inverse, the log2(P) steps that merge neighbouring groups
 * through the bridge blocks (twelve matrix maps and eight cross maps per
 * partition) and the production of every partition's blocks and bridges run
 * as one schedule on the whole GPU.  ``partitions`` must be a power of two,
 * at most n and at most 64 (pdiv_utils.py:16-81), else SINVB_EINVAL.
 * ``flags`` must be 0; the whole tridiagonal part of the inverse is written,
 * the bridges between partitions included.
 */
size_t sinvb_pdiv_workspace_size(int n, int b, int partitions, int dtype, unsigned flags);
int sinvb_pdiv_z(const void* diag, const void* upper, const void* lower, int n, int b, int partitions,
                 unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                 sinvb_stream_t stream);
int sinvb_pdiv_d(const void* diag, const void* upper, const void* lower, int n, int b, int partitions,
                 unsigned flags, void* G_diag, void* G_upper, void* G_lower, void* workspace, size_t workspace_bytes,
                 sinvb_stream_t stream);

/* ---- batched BCR: many independent matrices, levels in parallel -------------- */
/*
 * bcr_serial (src/sinv/algorithms/bcr/bcr_serial.py:19-62) over a batch of
 * matrices (descriptors as for the batched RGF; every instance may have its
 * own n and b).  Phase k of every matrix's reduction / production schedule
 * runs between the same two grid barriers, so the rows of a level of all
 * matrices are worked on by every SM at once.  ``status`` (optional, device,
 * ``count`` ints) gets each matrix's device status; ``flags`` is reserved (0).
 */
size_t sinvb_bcr_batched_workspace_size(const sinvb_batch_desc* descs, int count, int dtype, unsigned flags);
int sinvb_bcr_batched_z(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream);
int sinvb_bcr_batched_d(const sinvb_batch_desc* descs, int count, unsigned flags, void* workspace,
                        size_t workspace_bytes, int* status, sinvb_stream_t stream);
/*
 * Re-runs the batch last uploaded into ``workspace`` by sinvb_bcr_batched_*
 * with the same ``descs``: two memsets and one launch, no schedule building
 * and no host-to-device copy (capturable in a CUDA graph).
 */
int sinvb_bcr_batched_rerun_z(const sinvb_batch_desc* descs, int count, void* workspace, sinvb_stream_t stream);
int sinvb_bcr_batched_rerun_d(const sinvb_batch_desc* descs, int count, void* workspace, sinvb_stream_t stream);

/* ---- mixed-precision complex GEMM on the int8 tensor cores ---------------------- */
/*
 * No reference counterpart (the reference multiplies blocks with numpy/BLAS
 * zgemm, src/sinv/algorithms/rgf/rgf.py:48,53,60,62); the block product of
 * the mixed-precision sweeps, exposed on its own.  C = beta D + alpha A B for
 * row-major complex128 A (M x K), B (K x N), D, C (M x N), computed by the
 * Ozaki scheme on tcgen05.mma kind::i8: per-row / per-column power-of-two
 * scaling, `digits` signed 7-bit slices per value (1..8), exact int32
 * accumulation; error ~ 2^-(7*digits-1) relative to |A||B|.  D may be NULL.
 * Requires 2K <= 16384.
 */
size_t sinvb_zgemm_ozaki_workspace_size(int M, int N, int K, int digits);
int sinvb_zgemm_ozaki(int M, int N, int K, double alpha, const void* A, int lda, const void* B, int ldb,
                      double beta, const void* D, int ldd, void* C, int ldc, int digits, void* workspace,
                      size_t workspace_bytes, sinvb_stream_t stream);

/* ---- diagnostics ------------------------------------------------------------- */
/*
 * No reference counterpart: measures the FP64 tensor-core (DMMA) rate of the
 * current device, the ceiling of every FP64 kernel here (B200 has no FP64
 * kind of tcgen05.mma).  Runs `iters` dependent-free mma.sync.m8n8k4.f64
 * steps in 8 chains per warp, 8 warps per CTA, 2 CTAs per SM, timed with CUDA
 * events on `stream` (synchronises it).  Result in TFLOP/s.
 */
int sinvb_fp64_mma_peak(int iters, double* tflops, sinvb_stream_t stream);

/* ---- allocation-free variant ------------------------------------------------ */
/*
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they call (inside an allocator hook or host callback that must
 * not re-enter the allocator, or in a plugin whose host application owns all
 * device memory): the single-matrix complex128 RGF of sinvb_rgf_z with the
 * scratch in a static device array owned by the library (131,328 bytes, held
 * by every GPU that loads the library until exit), so only inputs and
 * outputs are passed.
 * Limits: b <= 64; SINVB_SAVE_OFFDIAG required when n > 1; flags other than
 * SINVB_SYM / SINVB_SAVE_OFFDIAG rejected (SINVB_EINVAL); output arrays that
 * overlap an input or each other rejected (SINVB_EINVAL).  ``status``
 * (optional, device, one int) receives the device status.  The first call on
 * a device does its set-up (the array's address, the kernels' shared-memory
 * attributes).  All calls share the array, so calls that overlap on the GPU
 * race.
 */
int sinvb_rgf_z_noalloc(const void* diag, const void* upper, const void* lower, int n, int b,
                        unsigned flags, void* G_diag, void* G_upper, void* G_lower, int* status,
                        sinvb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SINVB_H */
