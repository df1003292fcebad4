/*
 * swb_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the reference's Swift Alignment functions (swiftbwa,
 * Sources/Alignment/ Swift files and the BWACore/FMIndex pieces they use),
 * line for line, used only as the parity checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
 * (libswb_cuda.so) never links or calls it.
 *
 * Parity pin: every known-answer test of Tests/AlignmentTests/AlignmentTests.swift
 * that touches this path is replayed against this code by
 * tests/test_oracle_known_answers.py (fixtures in tests/golden/).  The Swift
 * reference itself cannot be built here (no Swift toolchain), so the pin is
 * those known answers plus the restatement's line-by-line citations.
 */
#ifndef SWB_ORACLE_H
#define SWB_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include "../include/swb_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Region produced by ExtensionAligner.extend (MemAlnReg subset,
 * Sources/BWACore/AlignmentRegion.swift:19-75). */
typedef struct orc_region {
    int64_t rb, re;
    int32_t qb, qe;
    int32_t rid, score, true_score, sub, sub_n, w, seed_cov, seed_len0;
} orc_region;

typedef struct orc_seed {   /* MemSeed (Sources/BWACore/Seed.swift) */
    int64_t rbeg;
    int32_t qbeg, len, score;
    int32_t pad;
} orc_seed;

void orc_scoring_matrix(const swb_scoring *sc, int8_t mat[25]);

/* BandedSWScalar.align -- Sources/Alignment/BandedSWScalar.swift:21-191 */
void orc_banded_sw_scalar(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                          const swb_scoring *sc, int32_t w, int32_t h0, int32_t end_bonus,
                          swb_ext_result *out, uint64_t *cells);
/* BandedSW16.align -- Sources/Alignment/BandedSW16.swift:8-203 */
void orc_banded_sw16(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                     const swb_scoring *sc, int32_t w, int32_t h0, swb_ext_result *out);
/* BandedSW8.align -- Sources/Alignment/BandedSW8.swift:10-213; returns 0 for nil */
int orc_banded_sw8(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                   const swb_scoring *sc, int32_t w, int32_t h0, swb_ext_result *out);

/* GlobalAligner.align -- Sources/Alignment/GlobalAligner.swift:19-232.
 * *n_cigar: in capacity, out ops.  Returns 0, or -1 when capacity is short
 * or w < 1 with qlen == tlen (the Swift code's 1...0 range). */
int orc_global_align(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                     const swb_scoring *sc, int32_t w, int32_t *score,
                     uint32_t *cigar, int32_t *n_cigar, uint64_t *cells);
/* GlobalAligner.computeNM -- GlobalAligner.swift:235-273 */
int32_t orc_compute_nm(const uint32_t *cigar, int32_t n, const uint8_t *q, int32_t qlen,
                       const uint8_t *t, int32_t tlen);

/* CIGARGenerator -- Sources/Alignment/CIGARGenerator.swift */
int32_t orc_infer_band_width(int32_t qlen, int32_t rlen, int32_t score, const swb_scoring *sc);
/* generate (:30-111).  md: NUL-terminated, md_cap bytes.  Returns 0 or -1. */
int orc_cigar_generate(const uint8_t *qseg, int32_t qlen, const uint8_t *rseg, int32_t rlen,
                       int32_t qb, int32_t qe, int32_t read_len, int32_t is_rev,
                       int32_t true_score, int32_t initial_w, const swb_scoring *sc,
                       int64_t ref_pos, uint32_t *cigar, int32_t *n_cigar,
                       int32_t *nm, char *md, int32_t md_cap, int32_t *score,
                       int64_t *pos, uint64_t *cells, int32_t *used_dp);
/* postProcess (:118-142) */
int orc_cigar_postprocess(const uint32_t *raw, int32_t n_raw, int32_t score,
                          const uint8_t *qseg, int32_t qlen, const uint8_t *rseg, int32_t rlen,
                          int32_t qb, int32_t qe, int32_t read_len, int32_t is_rev, int64_t ref_pos,
                          uint32_t *cigar, int32_t *n_cigar, int32_t *nm,
                          char *md, int32_t md_cap, int32_t *score_out, int64_t *pos);

/* LocalSWAligner.align -- Sources/Alignment/LocalSWAligner.swift:42-79.
 * Returns 1 with *out filled, or 0 for nil (out zeroed).  *path: 0 striped
 * u8, 1 scalar int32 fallback. */
int orc_local_align(const uint8_t *q, int32_t qlen, const uint8_t *t, int32_t tlen,
                    const swb_scoring *sc, int32_t min_sub_score,
                    swb_local_result *out, uint64_t *cells, int32_t *path);

/* PackedReference / FMIndex.getReference -- Sources/FMIndex/PackedReference.swift:34-55,
 * Sources/FMIndex/FMIndex.swift:147-170.  Returns bases written. */
uint8_t orc_pac_base(const uint8_t *pac, int64_t pos);
int32_t orc_get_reference(const uint8_t *pac, int64_t genome_len, int64_t pos, int32_t len,
                          uint8_t *buf);

/* ExtensionAligner.extend -- Sources/Alignment/ExtensionAligner.swift:114-346.
 * Reference access: ref_mode 0 = `ref` is an unpacked base array of
 * ref_len bases fetched with the tests' clamping closure
 * (Tests/AlignmentTests/AlignmentTests.swift:1097-1102); ref_mode 1 =
 * `ref` is a .pac and genome length ref_len, fetched with
 * FMIndex.getReference.  Returns number of regions (<= cap) or -1. */
int orc_extend(const orc_seed *seeds, int32_t n_seeds, int32_t rid,
               const uint8_t *read, int32_t read_len,
               const uint8_t *ref, int64_t ref_len, int32_t ref_mode,
               const swb_scoring *sc, orc_region *out, int32_t cap,
               uint64_t *sw_calls, uint64_t *cells);

/* Batch drivers over the ABI task structs (multi-threaded, static split).
 * pac/genome may be NULL when no task uses SWB_T_FROM_REF.  Return 0 or -1. */
int orc_ext_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                  uint64_t ref_bases, const swb_ext_task *tasks, size_t n,
                  swb_ext_result *out, int n_threads, uint64_t *cells);
int orc_global_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                     uint64_t ref_bases, const swb_global_task *tasks, size_t n,
                     swb_global_result *results, uint32_t *cigar_out, size_t cigar_cap,
                     int n_threads, uint64_t *cells);
int orc_cigar_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                    const swb_cigar_task *tasks, size_t n, swb_cigar_result *results,
                    uint32_t *cigar_out, size_t cigar_cap, char *md_out, size_t md_cap,
                    int n_threads, uint64_t *cells);
int orc_local_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac,
                    uint64_t ref_bases, const swb_local_task *tasks, size_t n,
                    swb_local_result *out, int n_threads, uint64_t *cells);

/* orc_extend (FMIndex.getReference targets) over many chains, in parallel:
 * chain c's regions go to out[seed_off ..] and their number to n_regions[c]. */
int orc_extend_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac, int64_t genome_len,
                     const swb_seed *seeds, const swb_chain *chains, size_t n_chains,
                     swb_region *out, uint32_t *n_regions, int n_threads, uint64_t *cells);

/* MateRescue.rescue (Sources/BWAMem/MateRescue.swift:29-171) for every job,
 * same layout as swb_mate_rescue; pac is the forward strand (.pac). */
int orc_mate_rescue_batch(const swb_scoring *sc, const uint8_t *bases, const uint8_t *pac, int64_t genome_len,
                          const swb_rescue_job *jobs, size_t n_jobs, const swb_anchor *templates,
                          const swb_anchor *mate_regions, const swb_orientation *stats, int32_t primary,
                          const int64_t *contig_offsets, const int32_t *contig_lengths, size_t n_contigs,
                          swb_rescued *out, uint32_t *n_out, uint32_t *n_cand, int n_threads, uint64_t *cells);

int orc_bwt_build(const uint8_t *codes, int64_t n, swb_bwt_checkpoint *cp, int64_t n_cp, int64_t count_out[5],
                  int64_t *length_out, int64_t *sentinel_out, int n_threads);
int64_t orc_smem_batch(const swb_bwt_checkpoint *cp, const int64_t count[5], int64_t length, int64_t sentinel,
                       const uint8_t *bases, const uint64_t *read_off, const int32_t *read_len, size_t n_reads,
                       int32_t min_seed_len, int64_t min_intv, int32_t split_len, int32_t split_width, uint32_t cap,
                       swb_smem *out, uint32_t *n_out, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
