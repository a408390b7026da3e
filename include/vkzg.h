/*
 * vkzg C API, implemented for one NVIDIA B200 (sm_100a) with hand-written CUDA.
 *
 * Drop-in replacement for jtraglia/vkzg's include/vkzg.h: the same symbols,
 * the same enum values, the same 4-byte options struct and the same buffer
 * layouts, so vkzg's Java FFM binding (bindings/java/.../Vkzg.java:118-135,
 * which looks symbols up by name and hard-codes sizeof(vkzg_options) == 4) and
 * any C caller link against this library unchanged.
 *
 * Every function is thread safe.  One vkzg_prover may be shared by many
 * threads; calls on one prover are serialised.  The caller owns all buffers;
 * the library copies inputs in and results out before returning and keeps no
 * pointer after a call.
 */
#ifndef VKZG_H
#define VKZG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ sizes
 * Reference: include/vkzg.h:31-37 */
#define VKZG_FIELD_ELEMENTS_PER_BLOB 4096
#define VKZG_NUM_CELL_PROOFS 128
#define VKZG_BYTES_PER_FIELD_ELEMENT 32
#define VKZG_BYTES_PER_BLOB (VKZG_FIELD_ELEMENTS_PER_BLOB * VKZG_BYTES_PER_FIELD_ELEMENT)
#define VKZG_BYTES_PER_PROOF 48
#define VKZG_FIELD_ELEMENTS_PER_CELL 64
#define VKZG_BYTES_PER_CELL (VKZG_FIELD_ELEMENTS_PER_CELL * VKZG_BYTES_PER_FIELD_ELEMENT)

/* ----------------------------------------------------------------- status
 * Reference: include/vkzg.h:41-49 (values are part of the ABI). */
typedef enum {
    VKZG_OK = 0,
    VKZG_ERR_BADARGS = 1,     /* null pointer, or a recovery blob with more than 64 cells missing */
    VKZG_ERR_MALLOC = 2,      /* host or device allocation failed */
    VKZG_ERR_IO = 3,          /* no setup tables or trusted setup could be read */
    VKZG_ERR_SETUP = 4,       /* a tables / setup file was malformed */
    VKZG_ERR_GPU = 5,         /* no CUDA device, or a CUDA call failed */
    VKZG_ERR_INVALID_BLOB = 6 /* a blob field element was not below the scalar modulus r */
} vkzg_result;

/* Human readable form of a status code; never NULL.
 * Replaces include/vkzg.h:52 (src/vkzg.cpp:170-181). */
const char *vkzg_error_string(vkzg_result r);

/* ---------------------------------------------------------------- options
 * Reference: include/vkzg.h:56-67.  Exactly one uint32_t. */
typedef struct {
    /* Blobs processed per device launch; larger calls are split into chunks of
     * this many.  About 4.5 MiB of device memory per blob.  0 = default (256). */
    uint32_t max_batch_size;
} vkzg_options;

/* Sets the defaults (max_batch_size = 0).  NULL-safe.  Replaces include/vkzg.h:70. */
void vkzg_options_default(vkzg_options *opts);

/* ----------------------------------------------------------------- prover */
typedef struct vkzg_prover vkzg_prover;

/*
 * Creates a prover on the current CUDA device.  Setup tables come from, in
 * order: $VKZG_TABLES_PATH (the reference's precomputed_tables.bin format,
 * src/precomputed_tables.cpp:16-58), precomputed_tables.bin next to this
 * library, or are generated on the GPU from the mainnet G1 monomial setup
 * ($VKZG_SETUP_PATH, else data/trusted_setup_g1_monomial.bin next to this
 * library).  Replaces include/vkzg.h:80 (src/vkzg.cpp:721-730).
 */
vkzg_result vkzg_prover_new(vkzg_prover **out, const vkzg_options *opts);

/* NULL-safe.  Replaces include/vkzg.h:82. */
void vkzg_prover_free(vkzg_prover *p);

/* CUDA device name, e.g. "NVIDIA B200"; "" for NULL.  Replaces include/vkzg.h:85. */
const char *vkzg_prover_device_name(const vkzg_prover *p);

/* Streaming multiprocessor count of the device (0 for NULL).  Replaces include/vkzg.h:88. */
uint32_t vkzg_prover_gpu_core_count(const vkzg_prover *p);

/* ---------------------------------------------------------------- compute */

/*
 * All 128 cell proofs of each of `num_blobs` consecutive blobs.
 * blobs:  num_blobs x 131072 bytes, 4096 big-endian canonical field elements.
 * proofs: num_blobs x 128 x 48 bytes, compressed G1, in cell (wire) order.
 * A non-canonical element anywhere in a chunk returns VKZG_ERR_INVALID_BLOB;
 * proofs of earlier chunks are already written.  num_blobs == 0 is a no-op.
 * Replaces include/vkzg.h:103-104 (src/vkzg.cpp:1183-1199).
 */
vkzg_result vkzg_compute_proofs_batch(vkzg_prover *p, uint8_t *proofs, const uint8_t *blobs,
                                      size_t num_blobs);

/*
 * Recovers all 128 cells of each of `num_blobs` consecutive blobs.
 * cells:        num_blobs x 128 x 2048 bytes, the extended blob in cell order;
 *               a missing cell's bytes are ignored, present cells are not
 *               canonicity-checked (values are taken mod r).
 * cell_present: num_blobs x 128 bytes, nonzero = present; at least 64 per blob,
 *               else VKZG_ERR_BADARGS (earlier chunks already written).
 * cells_out:    num_blobs x 128 x 2048 bytes, every cell.
 * Replaces include/vkzg.h:120-121 (src/vkzg.cpp:1201-1218).
 */
vkzg_result vkzg_recover_cells_batch(vkzg_prover *p, uint8_t *cells_out, const uint8_t *cells,
                                     const uint8_t *cell_present, size_t num_blobs);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* VKZG_H */
