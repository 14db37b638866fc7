// dsax_xengine -- the correlator stage as a ring-to-ring process, keeping the
// loop of src/dsaX_xgpu.cu (main, :150-357): connect to the input and output
// rings, copy the observation header through, then for every input block
// correlate it into the xGPU triangular visibility layout and write that to
// the output ring; a short input block ends the observation (:354-355).
// The reference promotes and calls xgpuCudaXengine per block; here one
// dsax_correlate call does the corner turn and the tcgen05 correlation, the
// ring buffers are pinned (cudaHostRegister, as src/dsaX_bfCorr.cu:86-114)
// so the copies are asynchronous DMA.  Errors are logged to stderr and end
// the process with EXIT_FAILURE, as the reference's stages do.
//   dsax_xengine -i IN_RING -o OUT_RING [-d DEVICE] [-t TIMEOUT_S]
// Header keys read (ASCII "KEY VALUE" lines): NPKT, NANT, NCHAN (defaults
// 2048, 63, 384).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dsax.h"
#include "dsax_ring.h"

static long header_int(const char *hdr, size_t n, const char *key, long dflt) {
  std::string h(hdr, n);
  const std::string k = std::string(key) + " ";
  size_t pos = 0;
  while ((pos = h.find(k, pos)) != std::string::npos) {
    if (pos == 0 || h[pos - 1] == '\n') return strtol(h.c_str() + pos + k.size(), nullptr, 10);
    pos += k.size();
  }
  return dflt;
}

int main(int argc, char **argv) {
  const char *in_name = nullptr, *out_name = nullptr;
  int device = 0;
  double timeout = 60.0;
  for (int i = 1; i + 1 < argc; i += 2) {
    if (!strcmp(argv[i], "-i")) in_name = argv[i + 1];
    else if (!strcmp(argv[i], "-o")) out_name = argv[i + 1];
    else if (!strcmp(argv[i], "-d")) device = atoi(argv[i + 1]);
    else if (!strcmp(argv[i], "-t")) timeout = atof(argv[i + 1]);
  }
  if (!in_name || !out_name) {
    fprintf(stderr, "usage: dsax_xengine -i IN_RING -o OUT_RING [-d DEVICE] [-t TIMEOUT_S]\n");
    return EXIT_FAILURE;
  }
  dsax_ring *rin = dsax_ring_connect(in_name, timeout);
  dsax_ring *rout = dsax_ring_connect(out_name, timeout);
  if (!rin || !rout) {
    fprintf(stderr, "dsax_xengine: could not connect to the rings\n");
    return EXIT_FAILURE;
  }
  std::vector<char> hdr(65536);
  uint64_t hn = 0;
  if (dsax_ring_read_header(rin, hdr.data(), hdr.size(), &hn) ||
      dsax_ring_write_header(rout, hdr.data(), hn)) {
    fprintf(stderr, "dsax_xengine: header exchange failed\n");
    return EXIT_FAILURE;
  }
  dsax_config cfg;
  dsax_default_config(&cfg);
  cfg.npkt = (int)header_int(hdr.data(), hn, "NPKT", cfg.npkt);
  cfg.nant_in = (int)header_int(hdr.data(), hn, "NANT", cfg.nant_in);
  cfg.nchan = (int)header_int(hdr.data(), hn, "NCHAN", cfg.nchan);
  const size_t block_bytes = dsax_block_bytes(&cfg, DSAX_FMT_CAPTURED);
  const size_t vis_bytes = dsax_vis_bytes(&cfg);
  if (dsax_ring_bufsz(rin) < block_bytes || dsax_ring_bufsz(rout) < vis_bytes) {
    fprintf(stderr, "dsax_xengine: ring blocks too small (%zu in, %zu out needed)\n", block_bytes,
            vis_bytes);
    return EXIT_FAILURE;
  }
  dsax_ctx *ctx = nullptr;
  int rc = dsax_create(&ctx, &cfg, device);
  if (rc != DSAX_OK) {
    fprintf(stderr, "dsax_xengine: dsax_create: %s\n", dsax_strerror(rc));
    return EXIT_FAILURE;
  }
  uint64_t tin = 0, tout = 0;
  char *din = dsax_ring_data(rin, &tin), *dout = dsax_ring_data(rout, &tout);
  const bool pin_in = dsax_register_host(ctx, din, tin) == DSAX_OK;
  const bool pin_out = dsax_register_host(ctx, dout, tout) == DSAX_OK;
  long blocks = 0;
  bool complete = false, failed = false;
  while (!complete && !failed) {
    uint64_t bytes = 0;
    char *blk = dsax_ring_open_read(rin, &bytes, nullptr);
    if (!blk) {
      fprintf(stderr, "dsax_xengine: input ring timed out\n");
      failed = true;
      break;
    }
    if (bytes >= block_bytes) {
      char *vis = dsax_ring_open_write(rout, nullptr);
      if (!vis) {
        fprintf(stderr, "dsax_xengine: output ring timed out\n");
        failed = true;
      } else if ((rc = dsax_correlate(ctx, blk, vis, DSAX_MEM_HOST)) != DSAX_OK) {
        fprintf(stderr, "dsax_xengine: block %ld: %s\n", blocks, dsax_last_error(ctx));
        failed = true;
      } else if (dsax_ring_close_write(rout, vis_bytes)) {
        failed = true;
      }
      ++blocks;
    }
    if (bytes < block_bytes) complete = true;   // short block: end of observation
    dsax_ring_close_read(rin);
  }
  // end of data downstream: one empty block
  if (!failed) {
    if (!dsax_ring_open_write(rout, nullptr) || dsax_ring_close_write(rout, 0)) failed = true;
  }
  if (pin_in) dsax_unregister_host(ctx, din);
  if (pin_out) dsax_unregister_host(ctx, dout);
  dsax_destroy(ctx);
  dsax_ring_disconnect(rin);
  dsax_ring_disconnect(rout);
  fprintf(stderr, "dsax_xengine: %ld blocks\n", blocks);
  return failed ? EXIT_FAILURE : EXIT_SUCCESS;
}
