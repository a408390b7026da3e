/*
 * vkzg CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A scalar CPU restatement of the reference's EIP-7594 hot path (jtraglia/vkzg):
 * BLS12-381 Fp/Fr Montgomery arithmetic, G1 Jacobian arithmetic, ZCash point
 * compression, the Fr NTTs, the FK20 cell-proof pipeline (phase A fixed-base
 * bucket MSM against the position table, doubling ladder, split-circulant
 * phase B, normalisation, compression) and cell recovery.  Every function
 * cites the reference file:line it follows.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product (libvkzg.so) never
 * links, loads or calls it.
 *
 * Parity is pinned by the consensus-spec vectors the reference ships
 * (tests/vectors/, converted to tests/golden/ by tests/golden/make_golden.py).
 */
#ifndef VKZG_ORACLE_H
#define VKZG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes mirror include/vkzg.h. */
enum { ORC_OK = 0, ORC_BADARGS = 1, ORC_MALLOC = 2, ORC_IO = 3, ORC_SETUP = 4, ORC_INVALID_BLOB = 6 };

typedef struct orc_tables orc_tables;

/* Builds the FK20 tables from 4096 compressed monomial G1 points ([tau^i]G1). */
int orc_tables_from_setup(orc_tables **out, const uint8_t *g1_monomial_compressed, int nthreads);
/* Loads / writes the reference's precomputed_tables.bin (format v1). */
int orc_tables_load(orc_tables **out, const char *path);
int orc_tables_write(const orc_tables *t, const char *path);
void orc_tables_free(orc_tables *t);
/* Raw views for tests: position table (262144 x 24 u32), roots, tap items. */
const uint32_t *orc_tables_position(const orc_tables *t);
size_t orc_tables_file_size(const orc_tables *t);
int orc_tables_serialize(const orc_tables *t, uint8_t *dst, size_t cap);

/* FK20 proofs, reference algorithm. proofs: n * 128 * 48 bytes. */
int orc_compute_proofs(const orc_tables *t, uint8_t *proofs, const uint8_t *blobs, size_t n, int nthreads);
/* FK20 proofs through plain G1 IFFT/truncate/FFT (independent phase-B form). */
int orc_compute_proofs_g1fft(const orc_tables *t, uint8_t *proofs, const uint8_t *blob);
/* Proofs straight from tau: [q_k(tau)]G1 with q_k = f div (X^64 - x_k).  tau: 32 B BE canonical. */
int orc_compute_proofs_tau(const uint8_t *tau_be, uint8_t *proofs, const uint8_t *blob);

/* Intermediate stages for kernel-level parity (all canonical, big-endian):
 * coeffs_f: 4096 x 32 B  polynomial coefficients (IFFT of the blob)
 * circ:     128 x 64 x 32 B  coeffs[j][i] (128-point FFT of circulant columns)
 * u:        128 x 96 B  phase-A outputs u[j], affine x||y (zeros = infinity)
 * proofs_nat: 128 x 96 B combined phase-B outputs in natural order, affine x||y */
int orc_proof_stages(const orc_tables *t, const uint8_t *blob, uint8_t *coeffs_f, uint8_t *circ,
                     uint8_t *u, uint8_t *proofs_nat);

/* Cell recovery, reference algorithm.  cells/cells_out: n * 128 * 2048 B; present: n * 128 B. */
int orc_recover_cells(uint8_t *cells_out, const uint8_t *cells, const uint8_t *present, size_t n,
                      int nthreads);
/* 128 cells (8192 x 32 B, wire order) of a blob: the 2x Reed-Solomon extension. */
int orc_compute_cells(uint8_t *cells, const uint8_t *blobs, size_t n, int nthreads);

/* Synthetic setup from a seed: tau (32 B BE), 4096 monomial and 4096 Lagrange (bit-reversed)
 * compressed G1 points.  Any output pointer may be NULL. */
int orc_synthetic_setup(uint64_t seed, uint8_t *tau_be, uint8_t *g1_monomial, uint8_t *g1_lagrange);

/* Field / curve primitives on canonical big-endian encodings (for known-answer tests). */
int orc_fp_mul_be(const uint8_t *a48, const uint8_t *b48, uint8_t *out48);
int orc_fr_mul_be(const uint8_t *a32, const uint8_t *b32, uint8_t *out32);
int orc_fr_inv_be(const uint8_t *a32, uint8_t *out32);
/* Montgomery limbs <-> canonical (Fp: 12 x u32 LE limbs; Fr: 8 x u32 LE limbs). */
void orc_fp_to_mont(const uint8_t *a48, uint32_t *mont12);
void orc_fp_from_mont(const uint32_t *mont12, uint8_t *a48);
void orc_fr_to_mont(const uint8_t *a32, uint32_t *mont8);
void orc_fr_from_mont(const uint32_t *mont8, uint8_t *a32);
/* G1: decompress 48 B -> affine x||y (96 B canonical BE), 0 on success. */
int orc_g1_decompress(const uint8_t *in48, uint8_t *xy96);
int orc_g1_compress(const uint8_t *xy96, uint8_t *out48);
/* k * P for a canonical scalar (32 B BE) and compressed point; writes compressed. */
int orc_g1_mul(const uint8_t *p48, const uint8_t *k32, uint8_t *out48);
/* Sum of compressed points. */
int orc_g1_add(const uint8_t *p48, const uint8_t *q48, uint8_t *out48);

#ifdef __cplusplus
}
#endif
#endif
