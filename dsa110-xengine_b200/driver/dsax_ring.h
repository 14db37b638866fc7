/* dsax_ring.h -- a psrdada-like block ring in POSIX shared memory, standing
 * in for the psrdada transport the reference's stages use (dada_hdu_* /
 * ipcbuf_* / ipcio_*, src/dsaX_xgpu.cu:180-357), which is not part of this
 * build.  One writer and one reader per ring.  A ring holds one header slot
 * (the ASCII observation header, up to hdrsz bytes) and nbufs data blocks of
 * bufsz bytes; a block closed with fewer than bufsz bytes ends the data
 * stream (the reader's "bytes_read < block_size" test).  Every wait is
 * bounded by a timeout (seconds) and returns an error when it expires. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dsax_ring dsax_ring;

/* Creates the shared-memory segment /name (fails if it exists). */
int dsax_ring_create(const char *name, uint64_t nbufs, uint64_t bufsz, uint64_t hdrsz);
int dsax_ring_destroy(const char *name);
dsax_ring *dsax_ring_connect(const char *name, double timeout_s);
void dsax_ring_disconnect(dsax_ring *r);

uint64_t dsax_ring_bufsz(const dsax_ring *r);
uint64_t dsax_ring_nbufs(const dsax_ring *r);
/* Start and length of the data blocks (to pin them with cudaHostRegister). */
char *dsax_ring_data(dsax_ring *r, uint64_t *total_bytes);

/* Header: written once by the writer, read once by the reader (blocks). */
int dsax_ring_write_header(dsax_ring *r, const char *hdr, uint64_t n);
int dsax_ring_read_header(dsax_ring *r, char *hdr, uint64_t cap, uint64_t *n);

/* Data blocks.  open_* return NULL on timeout or error. */
char *dsax_ring_open_write(dsax_ring *r, uint64_t *block_id);
int dsax_ring_close_write(dsax_ring *r, uint64_t bytes);
char *dsax_ring_open_read(dsax_ring *r, uint64_t *bytes, uint64_t *block_id);
int dsax_ring_close_read(dsax_ring *r);

#ifdef __cplusplus
}
#endif
