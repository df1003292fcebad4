/*
 * swb_cuda.h -- C ABI of the B200 (sm_100a) Smith-Waterman hot path of swiftbwa.
 *
 * This header is the drop-in boundary.  The Swift Alignment module keeps its
 * signatures; a maintainer adds this header next to
 * Sources/CHelpers/include/CHelpers.h (that target is already a C module
 * imported by Swift, Package.swift:55-58) and links libswb_cuda.so.  Every
 * entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Plain C: fixed-width integers, plain pointers and sizes.  No C++ or
 *     CUDA types cross the boundary.
 *   - The caller owns host buffers; the library owns device memory.
 *   - Every call returns an int status: SWB_OK (0) or a negative SWB_ERR_*
 *     code.  Nothing aborts or traps; swb_strerror() names the code and
 *     swb_last_error_message() carries detail for the calling thread.
 *   - A context is internally locked: concurrent calls from several host
 *     threads (Swift TaskGroup children) on one context are serialised.
 *   - Bases are 2-bit codes A=0 C=1 G=2 T=3, N=4, one byte per base
 *     (Sources/BWACore/Base.swift:2-44).  The resident reference is the
 *     bwa .pac layout: 4 bases per byte, first base in bits 7-6
 *     (Sources/FMIndex/PackedReference.swift:4-5,34-38).
 *   - Results are bit-exact with the reference's Swift CPU functions on the
 *     same inputs (scores, end coordinates, tie-breaks and CIGARs).
 */
#ifndef SWB_CUDA_H
#define SWB_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define SWB_OK                 0
#define SWB_ERR_INVALID_ARG   -1  /* null pointer, negative length, bad flag   */
#define SWB_ERR_NO_DEVICE     -2  /* no CUDA device / wrong architecture       */
#define SWB_ERR_CUDA          -3  /* a CUDA runtime call failed                 */
#define SWB_ERR_OOM           -4  /* allocation failed or over the memory budget */
#define SWB_ERR_TOO_LARGE     -5  /* a task exceeds the supported maximum size  */
#define SWB_ERR_NO_REFERENCE  -6  /* task reads the resident reference; none uploaded */
#define SWB_ERR_TIMEOUT       -7  /* a bounded device wait ran out              */
#define SWB_ERR_NOT_FOUND     -8  /* unknown ticket                             */
#define SWB_ERR_KERNEL        -9  /* a kernel reported an internal check failure */

/* --------------------------------------------------------------- scoring */
/* Mirrors the SW-relevant fields of ScoringParameters
 * (Sources/BWACore/ScoringParameters.swift:2-28).  The 5x5 matrix is
 * derived exactly as scoringMatrix() does (:65-73): a on the diagonal,
 * -b off it, -1 in any row or column of N. */
typedef struct swb_scoring {
    int32_t a;            /* matchScore                  (default 1)   */
    int32_t b;            /* mismatchPenalty             (default 4)   */
    int32_t o_ins;        /* gapOpenPenalty              (default 6)   */
    int32_t e_ins;        /* gapExtendPenalty            (default 1)   */
    int32_t o_del;        /* gapOpenPenaltyDeletion      (default 6)   */
    int32_t e_del;        /* gapExtendPenaltyDeletion    (default 1)   */
    int32_t zdrop;        /* zDrop                       (default 100) */
    int32_t pen_clip5;    /* penClip5                    (default 5)   */
    int32_t pen_clip3;    /* penClip3                    (default 5)   */
    int32_t band_width;   /* bandWidth                   (default 100) */
    int32_t min_seed_len; /* minSeedLength               (default 19)  */
} swb_scoring;

/* Fills *s with the defaults of ScoringParameters.init(). */
void swb_scoring_default(swb_scoring *s);

/* ------------------------------------------------------- task addressing */
/* A task names its query and target as spans of the caller's `bases`
 * buffer, or (target only) of the resident 2-bit reference.  Flags let
 * the kernel read a span reversed and/or complemented, so the left
 * extension's reversed prefix (ExtensionAligner.swift:209-224) and the
 * reverse-strand fetch (FMIndex.swift:147-163) need no host copies. */
#define SWB_Q_REVERSE   0x1u  /* query[j]  = bases[q_off + qlen-1-j]                 */
#define SWB_T_REVERSE   0x2u  /* target[i] = src[t_off + tlen-1-i]                   */
#define SWB_T_COMPLEMENT 0x4u /* target[i] = 3 - base for codes 0-3; N (4) stays N    */
#define SWB_T_FROM_REF  0x8u  /* target span is forward reference [t_off, t_off+tlen) */

/* ------------------------------------------------ kernel 1: banded extension */
/* Field order is SWResult's (Sources/BWACore/SWResult.swift:2-24). */
typedef struct swb_ext_result {
    int32_t score;    /* score            */
    int32_t qle;      /* queryEnd         */
    int32_t tle;      /* targetEnd        */
    int32_t gtle;     /* globalTargetEnd  */
    int32_t gscore;   /* globalScore      */
    int32_t max_off;  /* maxOff           */
} swb_ext_result;

/* One call of BandedSWScalar.align(query:target:scoring:w:h0:endBonus:)
 * (Sources/Alignment/BandedSWScalar.swift:21-28). */
typedef struct swb_ext_task {
    uint64_t q_off;      /* query span start in `bases`                      */
    uint64_t t_off;      /* target span start in `bases` or the reference    */
    int32_t  qlen;       /* query length  (0 -> all-zero result, :33-35)      */
    int32_t  tlen;       /* target length (0 -> all-zero result)              */
    int32_t  w;          /* band width                                        */
    int32_t  h0;         /* initial score                                     */
    int32_t  end_bonus;  /* endBonus                                          */
    uint32_t flags;      /* SWB_Q_REVERSE | SWB_T_*                           */
} swb_ext_task;          /* 40 bytes */

/* ---------------------------------------- kernel 2: banded global + CIGAR */
/* One call of GlobalAligner.align(query:target:scoring:w:scoringMatrix:)
 * (Sources/Alignment/GlobalAligner.swift:19-25); with true_score set and
 * SWB_GLB_RETRY it also runs CIGARGenerator.generate's band-doubling retry
 * (CIGARGenerator.swift:88-96) on the device. */
#define SWB_GLB_RETRY 0x100u
typedef struct swb_global_task {
    uint64_t q_off, t_off;
    int32_t  qlen, tlen;
    int32_t  w;           /* band width (GlobalAligner's `w`)                 */
    int32_t  true_score;  /* retry while score < true_score (SWB_GLB_RETRY)   */
    uint32_t flags;       /* SWB_Q_REVERSE | SWB_T_* | SWB_GLB_RETRY          */
    int32_t  reserved;
} swb_global_task;        /* 40 bytes */

/* CIGAR ops are packed (len << 4) | op, op M=0 I=1 D=2 S=4 H=5
 * (Sources/Alignment/CIGARBuilder.swift:4-37). */
typedef struct swb_global_result {
    int32_t  score;       /* h[qlen] of the last attempt (GlobalAligner.swift:144) */
    int32_t  n_cigar;     /* ops written at cigar + cigar_off                       */
    int32_t  w_used;      /* band width of the last attempt                         */
    int32_t  attempts;    /* 1 + retries                                             */
    uint64_t cigar_off;   /* offset (in ops) of this task's CIGAR in the output      */
} swb_global_result;

/* One call of CIGARGenerator.generate(querySegment:refSegment:qb:qe:readLength:
 * isReverse:trueScore:initialW:scoring:refPos:) (CIGARGenerator.swift:30-111):
 * band inference, the pure-M fast path, banded global alignment with the
 * band-doubling retry, leading/trailing deletion squeeze, NM, MD and soft
 * clips.  q_off/qlen is the query segment, t_off/rlen the reference segment
 * (spans as for the other tasks; SWB_T_* flags apply to the segment). */
typedef struct swb_cigar_task {
    uint64_t q_off, t_off;
    int32_t  qlen, rlen;
    int32_t  qb, qe;          /* alignment bounds in read coordinates        */
    int32_t  read_len;
    int32_t  is_reverse;
    int32_t  true_score;
    int32_t  initial_w;
    int64_t  ref_pos;
    uint32_t flags;
    int32_t  reserved;
} swb_cigar_task;             /* 64 bytes */

/* CIGARResult (Sources/Alignment/GlobalAlignResult.swift:20-44).  The CIGAR
 * (soft clips included) is at cigar_out[cigar_off .. +n_cigar), the MD
 * string (NUL-terminated) at md_out[md_off]. */
typedef struct swb_cigar_result {
    int32_t  score;
    int32_t  nm;
    int32_t  n_cigar;
    int32_t  md_len;
    int64_t  pos;
    uint64_t cigar_off;       /* sum over earlier tasks of (qlen + rlen + 2)       */
    uint64_t md_off;          /* sum over earlier tasks of (6 * (qlen + rlen) + 8) */
    int32_t  used_dp;         /* 0 = pure-M fast path (:59-80), 1 = global DP      */
    int32_t  reserved;
} swb_cigar_result;           /* 48 bytes */

/* ------------------------------------------------ kernel 3: local SW (rescue) */
/* One call of LocalSWAligner.align(query:target:scoring:scoringMatrix:minSubScore:)
 * (Sources/Alignment/LocalSWAligner.swift:42-45). */
typedef struct swb_local_task {
    uint64_t q_off, t_off;
    int32_t  qlen, tlen;
    int32_t  min_sub_score; /* clamped to 0..255 like UInt8(clamping:) (MateRescue.swift:125) */
    uint32_t flags;
} swb_local_task;           /* 32 bytes */

/* LocalSWResult (LocalSWAligner.swift:4-23).  The Swift function returns
 * nil exactly when score == 0 here. */
typedef struct swb_local_result {
    int32_t score;
    int32_t qb, qe;   /* queryBegin, queryEnd (inclusive)   */
    int32_t tb, te;   /* targetBegin, targetEnd (inclusive) */
    int32_t score2;
} swb_local_result;

/* ------------------------------------------------------------------ context */
typedef struct swb_ctx swb_ctx;

/* Replaces MetalSWEngine.shared (Sources/MetalSW/MetalSWEngine.swift:8-17):
 * binds `device`, creates the context's stream, and caps the library's
 * device allocations at mem_budget_bytes (0 = 3/4 of free memory). */
int  swb_init(int device, size_t mem_budget_bytes, swb_ctx **out);
void swb_destroy(swb_ctx *ctx);
const char *swb_strerror(int status);
/* Detail of the last failing call on this host thread ("" if none). */
const char *swb_last_error_message(void);

/* Keeps the forward strand resident in HBM in .pac layout
 * (PackedReference.swift:4-55).  n_bases bases, (n_bases+3)/4 bytes. */
int swb_upload_reference(swb_ctx *ctx, const uint8_t *pac, uint64_t n_bases);

/* ------------------------------------------------ synchronous batch entry points */
/* Host buffers in, host results out.  Replaces
 * BandedSWDispatcher.dispatchBatch8/dispatchBatch16
 * (Sources/MetalSW/BandedSWDispatcher.swift:48,107); unlike those, one call
 * returns exact results for every task (no nil, no caller-side rerun). */
int swb_ext_batch(swb_ctx *ctx, const swb_scoring *sc,
                  const uint8_t *bases, size_t n_bases,
                  const swb_ext_task *tasks, size_t n_tasks,
                  swb_ext_result *out);

/* Replaces GlobalSWDispatcher.dispatchBatch (GlobalSWDispatcher.swift:40).
 * cigar_out receives every task's ops; results[i].cigar_off indexes it.
 * cigar_cap must be >= sum over tasks of (qlen + tlen). */
int swb_global_batch(swb_ctx *ctx, const swb_scoring *sc,
                     const uint8_t *bases, size_t n_bases,
                     const swb_global_task *tasks, size_t n_tasks,
                     swb_global_result *results,
                     uint32_t *cigar_out, size_t cigar_cap);

/* CIGARGenerator.generate for a batch (replaces the GlobalSWDispatcher +
 * CIGARGenerator.postProcess pair of BWAMemAligner.swift:483-668).
 * cigar_cap >= sum of (qlen + rlen + 2); md_cap >= sum of (6*(qlen+rlen)+8).
 * Bases and tasks in pinned host memory (cudaHostAlloc / registered) are
 * copied straight to the device; pageable ones go through the context's
 * pinned staging buffer.  Likewise results, cigar_out and md_out: when all
 * three are pinned the device writes them directly, else through pinned
 * staging and host threads. */
int swb_cigar_batch(swb_ctx *ctx, const swb_scoring *sc,
                    const uint8_t *bases, size_t n_bases,
                    const swb_cigar_task *tasks, size_t n_tasks,
                    swb_cigar_result *results,
                    uint32_t *cigar_out, size_t cigar_cap,
                    char *md_out, size_t md_cap);

/* Replaces LocalSWDispatcher.dispatchBatch (LocalSWDispatcher.swift:31),
 * with score2 computed on the device (the Metal path hard-codes it to 0,
 * BWAMemAligner.swift:1942). */
int swb_local_batch(swb_ctx *ctx, const swb_scoring *sc,
                    const uint8_t *bases, size_t n_bases,
                    const swb_local_task *tasks, size_t n_tasks,
                    swb_local_result *out);

/* ------------------------------------- device-resident entry point (HBM in/out) */
/* Same as swb_ext_batch with every pointer a device pointer on the
 * context's device, enqueued on `stream` (a cudaStream_t, NULL = the
 * context's stream); returns without synchronising. */
int swb_ext_batch_device(swb_ctx *ctx, const swb_scoring *sc,
                         const uint8_t *d_bases, const swb_ext_task *d_tasks,
                         size_t n_tasks, swb_ext_result *d_out, void *stream);

/* The plain one-launch-per-batch form of swb_ext_batch_device, the dispatch
 * shape of BandedSWDispatcher.dispatchBatch8/16 (BandedSWDispatcher.swift:48,107):
 * one launch over the batch in input order, one task per thread, with the
 * same two-row kernel code as the binned pass and rows sized for the
 * batch's longest query (int8 rows when every task's scores fit a byte,
 * else int16) -- no sort, no length bins, no claiming.  Tasks that code
 * cannot take (queries above 256 bases, scores beyond int16) run the
 * binned pass's int32 kernels afterwards.  Same results as
 * swb_ext_batch_device; it exists as the baseline that batching is
 * measured against.  Reads the batch's shape back from the device, so it
 * synchronises `stream` once before its main launch. */
int swb_ext_batch_plain_device(swb_ctx *ctx, const swb_scoring *sc,
                               const uint8_t *d_bases, const swb_ext_task *d_tasks,
                               size_t n_tasks, swb_ext_result *d_out, void *stream);

/* Length classes of the extension bins: ascending bounds on the row length
 * a task keeps, min(qlen, 2w + 2) with w the band after the reference's
 * clamp (BandedSWScalar.swift:52-62) -- a band narrower than the query is
 * kept as a ring of its columns -- as 1..15 values within [8, 256]; each
 * class has an int8-row and an int16-row bin (two target rows per pass, one
 * task per thread), and rows above the last bound, or scores beyond int16,
 * run one warp per extension.  Defaults: 32 48 64 80 96 112 128 160 192 256.
 * No reference counterpart: the reference dispatches every batch to one
 * kernel (BandedSWDispatcher.swift:48,107). */
int swb_set_ext_bins(swb_ctx *ctx, const int32_t *qmax, int n);
int swb_get_ext_bins(swb_ctx *ctx, int32_t *qmax, int cap, int *n);
/* Autotuner: times candidate class sets (the defaults, uniform steps, and
 * quantiles of the batch's row lengths and estimated cells) on the given
 * sample batch (host arrays, as swb_ext_batch; best of two runs after a
 * warm-up each) and keeps the fastest in the context, the defaults unless
 * another set is more than 2 % faster.  Writes the chosen classes
 * (qmax_out[0..cap), *n_out), the chosen set's and the defaults' time on
 * the sample (ms; may be NULL). */
int swb_tune_ext_bins(swb_ctx *ctx, const swb_scoring *sc, const uint8_t *bases, size_t n_bases,
                      const swb_ext_task *tasks, size_t n_tasks, int32_t *qmax_out, int cap, int *n_out,
                      float *best_ms, float *default_ms);

/* Allocation-free variant of swb_ext_batch_device.  It has no counterpart
 * in the reference.  It is for callers that cannot let a library call
 * cudaMalloc: a server whose own arena already holds the free HBM (the
 * resident reference and admitted request buffers), or a continuous-batching
 * loop that cannot afford cudaMalloc/cudaFree stalling its other streams.
 * It needs no context: it runs on the calling thread's current device and
 * on `stream` (a cudaStream_t, NULL = the legacy default stream); every
 * pointer is a device pointer the caller owns (d_pac: the .pac reference
 * for SWB_T_FROM_REF spans, may be NULL otherwise; spans are trusted, as in
 * swb_ext_batch_device).  Its only working memory is one static device
 * array of 18.9 MB.  A GPU holds it from the first call on that GPU (which
 * loads this code there under CUDA's default lazy module loading; a call
 * with n_tasks = 0 is enough) until the process exits, so a caller that is
 * about to hand the free HBM to its own arena makes that first call before.
 * Limit: a task that needs the int32 path (query above 256 bases, or
 * h0 + qlen*maxScore above 32000) may have at most 1024 query bases; a
 * longer one gets an all-zero result and the call returns
 * SWB_ERR_TOO_LARGE naming the first such task.  The first call on a device
 * does a one-time set-up (looks up the array's address, sizes a kernel), so
 * make that first call before any stream capture.  Every call synchronises
 * `stream` to read its status words.  Calls share the array: calls from threads of one
 * process take turns (a per-device lock held until the stream is done);
 * calls from different processes on one GPU that overlap there race. */
int swb_ext_batch_static(const swb_scoring *sc, const uint8_t *d_bases, const uint8_t *d_pac,
                         const swb_ext_task *d_tasks, size_t n_tasks, swb_ext_result *d_out,
                         void *stream);

/* ------------------------------------------ extension driver (whole chains) */
/* MemSeed (Sources/BWACore/Seed.swift): rbeg in BWT coordinates
 * [0, 2*genome_len). */
typedef struct swb_seed {
    int64_t rbeg;
    int32_t qbeg, len, score;
    int32_t reserved;
} swb_seed;                 /* 24 bytes */

/* One chain: seeds[seed_off .. seed_off+n_seeds) of the read
 * bases[read_off .. read_off+read_len). */
typedef struct swb_chain {
    uint64_t read_off;
    int32_t  read_len;
    int32_t  rid;
    uint32_t seed_off, n_seeds;
} swb_chain;                /* 24 bytes */

/* MemAlnReg fields ExtensionAligner.extend sets (AlignmentRegion.swift:19-75). */
typedef struct swb_region {
    int64_t rb, re;
    int32_t qb, qe;
    int32_t rid, score, true_score, sub, sub_n, w, seed_cov, seed_len0;
} swb_region;               /* 56 bytes */

/* ExtensionAligner.extend for many chains at once
 * (Sources/Alignment/ExtensionAligner.swift:114-346), with targets fetched
 * from the resident reference as FMIndex.getReference does
 * (Sources/FMIndex/FMIndex.swift:147-170; the uploaded reference is the
 * forward strand of length genome_len).  Chains advance in rounds: each
 * round extends the next pending seed of every active chain on the GPU
 * (left, its band retry, right, its band retry), so the covered-region
 * skip, the retries and the left-to-right h0 chaining are the reference's.
 * Chain c's regions are out[seed_off .. seed_off + n_regions[c]) (at most
 * one region per seed).  *rounds (optional) receives the GPU batches run.
 * Inputs (bases, seeds, chains) and outputs (out, n_regions) in pinned host
 * memory are copied straight to and from the device; pageable ones go
 * through the context's pinned staging buffer and host threads. */
int swb_extend_chains(swb_ctx *ctx, const swb_scoring *sc,
                      const uint8_t *bases, size_t n_bases,
                      const swb_seed *seeds, size_t n_seeds,
                      const swb_chain *chains, size_t n_chains, uint64_t genome_len,
                      swb_region *out, uint32_t *n_regions, uint32_t *rounds);

/* ------------------------------------------------ mate rescue (MateRescue.swift) */
/* Insert-size statistics of one pair orientation, the fields mate rescue
 * reads (OrientationStats, Sources/BWAMem/InsertSizeEstimator.swift:21-35).
 * Orientations are indexed FF 0, FR 1, RF 2, RR 3. */
typedef struct swb_orientation {
    int32_t failed;           /* nonzero: orientation skipped */
    int32_t reserved;
    int64_t proper_low, proper_high;
} swb_orientation;           /* 24 bytes */

/* The two MemAlnReg fields rescue reads from template and mate regions. */
typedef struct swb_anchor {
    int64_t rb;               /* BWT coordinate, [0, 2*genome_len) */
    int32_t rid;
    int32_t reserved;
} swb_anchor;                /* 16 bytes */

/* One MateRescue.rescue call: the mate read bases[mate_off ..+mate_len),
 * its template regions templates[tmpl_off ..+n_tmpl) and the mate's own
 * regions mate_regions[mreg_off ..+n_mreg). */
typedef struct swb_rescue_job {
    uint64_t mate_off;
    int32_t  mate_len;
    int32_t  reserved;
    uint32_t tmpl_off, n_tmpl;
    uint32_t mreg_off, n_mreg;
} swb_rescue_job;            /* 32 bytes */

/* A rescued region: the MemAlnReg fields MateRescue sets (MateRescue.swift:
 * 133-163); the others keep MemAlnReg() defaults (sub 0, subN 0, w 0,
 * secondary -1, seedLen0 0). */
typedef struct swb_rescued {
    int64_t rb, re;
    int32_t qb, qe;
    int32_t rid, score, true_score, csub, seed_cov, reserved;
} swb_rescued;               /* 48 bytes */

/* MateRescue.rescue (Sources/BWAMem/MateRescue.swift:29-171) for many
 * mates: for each template region and each non-failed orientation without a
 * consistent mate hit, the rescue window is clamped, fetched from the
 * resident reference strand-aware within the template's contig
 * (PackedReference.fetchSequence, PackedReference.swift:73-121), aligned
 * with LocalSWAligner.align (minSubScore = UInt8(clamping: min_seed_len*a))
 * and kept when score >= min_seed_len*a.  Contigs are given by their
 * offsets (ascending) and lengths in the forward strand (ReferenceMetadata
 * annotations).  Job j's regions are out[4*tmpl_off ..+n_out[j]), in the
 * reference's order; out must hold 4*n_templates entries.  n_cand (optional)
 * receives the local alignments run per job. */
int swb_mate_rescue(swb_ctx *ctx, const swb_scoring *sc,
                    const uint8_t *bases, size_t n_bases,
                    const swb_rescue_job *jobs, size_t n_jobs,
                    const swb_anchor *templates, size_t n_templates,
                    const swb_anchor *mate_regions, size_t n_mate_regions,
                    const swb_orientation stats[4], int32_t primary_orientation,
                    const int64_t *contig_offsets, const int32_t *contig_lengths, size_t n_contigs,
                    uint64_t genome_len, swb_rescued *out, uint32_t *n_out, uint32_t *n_cand);

/* ------------------------------------------------ SMEM seeding (FM index) */
/* CheckpointOCC (Sources/FMIndex/CheckpointOCC.swift:6-13): the cumulative
 * A, C, G, T counts before a block of 64 BWT characters and one bitstring
 * per base with bit 63-y set when position y of the block holds it. */
typedef struct swb_bwt_checkpoint {
    int64_t  counts[4];
    uint64_t bits[4];
} swb_bwt_checkpoint;        /* 64 bytes */

/* SMEM (Sources/BWACore/SMEM.swift:5-29): SA interval [k, l], inclusive,
 * and the query span [qb, qe). */
typedef struct swb_smem {
    int64_t k, l;
    int32_t qb, qe;
} swb_smem;                  /* 24 bytes */

/* Keeps the BWT resident in HBM (the fields of BWT, Sources/FMIndex/BWT.swift:5-20):
 * n_cp = (length >> 6) + 1 checkpoints, count[5] = the cumulative base
 * counts each +1 for the sentinel (count[4] = length), sentinel = the BWT
 * position of '$'.  Replaces the Metal engine's bwtCheckpointBuffer /
 * bwtCountsBuffer / bwtSentinelBuffer (MetalSWEngine.swift:88-120). */
int swb_upload_bwt(swb_ctx *ctx, const swb_bwt_checkpoint *cp, uint64_t n_cp, const int64_t count[5],
                   int64_t length, int64_t sentinel);

/* SMEMFinder.findAllSMEMs(query:bwt:minSeedLen:minIntv:) (SMEMFinder.swift:28-63)
 * for many reads on the resident BWT, followed, when split_len > 0, by the
 * internal re-seeding of BWAMemAligner.internalReseed (BWAMemAligner.swift:259-305):
 * every SMEM at least split_len long with at most split_width occurrences is
 * searched again from its midpoint with minIntv = its count + 1 and the new
 * SMEMs join the list (split_len = Int(Float(minSeedLength) * seedSplitRatio
 * + 0.499) as the reference computes it, 28 for the defaults; split_width =
 * splitWidth, 10).  Read r is bases[read_off[r] ..+ read_len[r])
 * (codes 0-4, N = 4).  Its n_out[r] SMEMs, sorted by query begin then
 * longest first, are out[out_off[r] ..+ n_out[r]] (out_off = the running
 * sum of n_out, so the reads' lists are packed in read order); out holds
 * out_cap entries.  cap_per_read bounds the SMEMs of one read the device
 * keeps while it searches.  When a read has more than cap_per_read SMEMs,
 * n_out[r] still counts them all, only the first cap_per_read found (in
 * the order found) are written at its offset, and the call returns
 * SWB_ERR_TOO_LARGE naming the first such read; when the total exceeds
 * out_cap the call returns SWB_ERR_TOO_LARGE with n_out and out_off filled
 * and nothing written to out.  Either way the caller can retry with larger
 * bounds, and every other read's results are complete.  At most 2^31-16
 * reads per call.  Inputs (bases, read_off, read_len) and outputs (out,
 * n_out, out_off) in pinned host memory are copied straight to and from the
 * device; pageable ones go through pinned staging and host threads.  Replaces
 * the CPU loop of BWAMemAligner.alignReadPhase1to3 (BWAMemAligner.swift:133-139)
 * and the Metal forward kernel (Kernels/smem_forward.metal:117) for a batch. */
int swb_smem_batch(swb_ctx *ctx, const uint8_t *bases, size_t n_bases, const uint64_t *read_off,
                   const int32_t *read_len, size_t n_reads, int32_t min_seed_len, int64_t min_intv,
                   int32_t split_len, int32_t split_width, uint32_t cap_per_read, swb_smem *out, size_t out_cap,
                   uint32_t *n_out, uint64_t *out_off);

/* ------------------------------------------------ serving (continuous batching) */
/* A request loop over one context's GPU for extension batches of differing
 * sizes that arrive concurrently (the actor loop of BWAMemAligner's
 * read-chunk pipeline, main.swift:315-423, batching its extensions).
 * Requests are queued and answered asynchronously by ticket.  A worker
 * thread forms waves from the head of the queue (at most max_wave_tasks
 * tasks, large requests split across waves so small ones do not wait behind
 * them), stages each request's bases once into a device arena admitted
 * against arena_bytes, sorts/bins every wave's tasks together, and
 * rotates waves over three internal lanes so that one wave's copies
 * overlap the other's kernels.  plain = 1 disables all of that: one
 * request at a time, one launch sequence each (the baseline).  The caller
 * keeps each request's buffers alive until its ticket completes; each
 * task's result is the same as from swb_ext_batch. */
typedef struct swb_server swb_server;
typedef struct swb_server_opts {
    size_t   arena_bytes;      /* device bytes for request bases (0 = 1 GiB)   */
    size_t   max_wave_tasks;   /* tasks per wave (0 = 1M)                      */
    int32_t  plain;            /* 0 = served (waves, three lanes); 1 = one request
                                  at a time through the binned launch sequence;
                                  2 = one request at a time through the plain
                                  one-launch-per-batch kernel
                                  (swb_ext_batch_plain_device)                 */
    int32_t  start_paused;     /* 1 = admit nothing until swb_server_resume    */
    uint32_t latency_cells;    /* served mode: tasks with more DP cells than this
                                  (qlen * tlen) run one warp per extension, so no
                                  single long task holds a wave open; 0 = off  */
    uint32_t reserved;
} swb_server_opts;
typedef struct swb_server_stats {
    uint64_t submitted, completed, tasks_completed, waves;
    uint64_t cells;            /* DP cells of completed waves                  */
    double   busy_ms;          /* summed wave device time                      */
} swb_server_stats;
int swb_server_start(swb_ctx *ctx, const swb_scoring *sc, const swb_server_opts *opts, swb_server **out);
/* Task offsets (q_off, and t_off of spans not in the reference) are
 * relative to bases - span_origin: the byte a task addresses as x is
 * bases[x - span_origin], so a request can be a slice of a larger pool
 * without rebasing.  Pinned (cudaHostAlloc/registered) bases, tasks and out
 * are copied asynchronously with no host-side pass; pageable ones work too,
 * through bounce buffers. */
int swb_server_submit(swb_server *srv, const uint8_t *bases, size_t n_bases, uint64_t span_origin,
                      const swb_ext_task *tasks, size_t n_tasks, swb_ext_result *out, uint64_t *ticket);
/* *done = 1 once the ticket completed; *status = its result status. */
int swb_server_poll(swb_server *srv, uint64_t ticket, int *done, int *status);
/* Waits at most timeout_ms (SWB_ERR_TIMEOUT after that).  On completion the
 * ticket is released and its submit/completion times (steady-clock ns) are
 * returned; *status is the request's own status. */
int swb_server_wait(swb_server *srv, uint64_t ticket, int timeout_ms, int *status,
                    uint64_t *submit_ns, uint64_t *done_ns);
int swb_server_resume(swb_server *srv);
int swb_server_stats_get(swb_server *srv, swb_server_stats *st);
/* Drains the queue, stops the worker, frees the server's device memory. */
int swb_server_stop(swb_server *srv);

/* --------------------------------------------- single-call Swift signatures */
/* BandedSWScalar.align (BandedSWScalar.swift:21-28). */
int swb_banded_sw_align(swb_ctx *ctx, const uint8_t *query, int32_t qlen,
                        const uint8_t *target, int32_t tlen,
                        const swb_scoring *sc, int32_t w, int32_t h0,
                        int32_t end_bonus, swb_ext_result *out);
/* GlobalAligner.align (GlobalAligner.swift:19-25).  *n_cigar in: capacity
 * of cigar (>= qlen + tlen), out: ops written. */
int swb_global_align(swb_ctx *ctx, const uint8_t *query, int32_t qlen,
                     const uint8_t *target, int32_t tlen,
                     const swb_scoring *sc, int32_t w,
                     int32_t *score, uint32_t *cigar, int32_t *n_cigar);
/* LocalSWAligner.align (LocalSWAligner.swift:42-45); out->score == 0 <=> nil. */
int swb_local_align(swb_ctx *ctx, const uint8_t *query, int32_t qlen,
                    const uint8_t *target, int32_t tlen,
                    const swb_scoring *sc, int32_t min_sub_score,
                    swb_local_result *out);

/* ------------------------------------------------------- library introspection */
/* Per-kernel accounting.  With profiling on, every kernel launch is
 * bracketed by CUDA events on its stream; swb_profile_read synchronises the
 * context's streams and returns, per kernel name, the launches, summed
 * device time and DP cells since the last swb_profile_reset. */
typedef struct swb_kernel_stat {
    char     name[40];
    uint32_t launches;
    double   total_ms;
    uint64_t cells;
} swb_kernel_stat;
int swb_profile(swb_ctx *ctx, int enable);
int swb_profile_reset(swb_ctx *ctx);
int swb_profile_read(swb_ctx *ctx, swb_kernel_stat *stats, int cap, int *n_stats);
/* Measured int32 add+max issue rate of the context's GPU (ops/s): the
 * denominator of the kernels' integer-ALU roofline. */
int swb_int_alu_peak(swb_ctx *ctx, double *ops_per_s);
/* Measured packed-16-bit (s16x2 DPX add+max) rate of the context's GPU, in
 * 16-bit lane operations/s: the int16 roofline of the two-row kernel. */
int swb_int16x2_alu_peak(swb_ctx *ctx, double *lane_ops_per_s);

/* Kernel launches issued by this context so far (for launch accounting). */
uint64_t swb_kernel_launches(const swb_ctx *ctx);
/* Device time (ms, CUDA events on the context's stream) of the last
 * synchronous batch call's kernels, and DP cells it updated. */
int swb_last_batch_stats(const swb_ctx *ctx, double *kernel_ms, uint64_t *cells);

#ifdef __cplusplus
}
#endif
#endif /* SWB_CUDA_H */
