// dsax_ringtool -- create, fill and drain dsax_ring segments (for feeding the
// driver from files and collecting its output).
//   dsax_ringtool create NAME NBUFS BUFSZ [HDRSZ]
//   dsax_ringtool destroy NAME
//   dsax_ringtool put NAME FILE [HEADER_FILE]   file -> blocks, then end of data
//   dsax_ringtool get NAME FILE                 blocks -> file until end of data
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dsax_ring.h"

static int usage() {
  fprintf(stderr,
          "usage: dsax_ringtool create NAME NBUFS BUFSZ [HDRSZ] | destroy NAME |\n"
          "       put NAME FILE [HEADER_FILE] | get NAME FILE\n");
  return 2;
}

int main(int argc, char **argv) {
  if (argc < 3) return usage();
  const char *cmd = argv[1], *name = argv[2];
  if (!strcmp(cmd, "create")) {
    if (argc < 5) return usage();
    const uint64_t hdrsz = argc > 5 ? strtoull(argv[5], nullptr, 10) : 4096;
    const int rc = dsax_ring_create(name, strtoull(argv[3], nullptr, 10),
                                    strtoull(argv[4], nullptr, 10), hdrsz);
    if (rc) fprintf(stderr, "create %s failed (%d)\n", name, rc);
    return rc ? 1 : 0;
  }
  if (!strcmp(cmd, "destroy")) return dsax_ring_destroy(name) ? 1 : 0;
  if (argc < 4) return usage();
  dsax_ring *r = dsax_ring_connect(name, 120.0);
  if (!r) {
    fprintf(stderr, "cannot connect to %s\n", name);
    return 1;
  }
  const uint64_t bufsz = dsax_ring_bufsz(r);
  int rc = 0;
  if (!strcmp(cmd, "put")) {
    std::vector<char> hdr(4096, 0);
    uint64_t hn = 0;
    if (argc > 4) {
      FILE *hf = fopen(argv[4], "rb");
      if (!hf) return 1;
      hn = fread(hdr.data(), 1, hdr.size(), hf);
      fclose(hf);
    }
    if (dsax_ring_write_header(r, hdr.data(), hn)) return 1;
    FILE *f = fopen(argv[3], "rb");
    if (!f) return 1;
    for (;;) {
      char *b = dsax_ring_open_write(r, nullptr);
      if (!b) { rc = 1; break; }
      const size_t n = fread(b, 1, bufsz, f);
      if (dsax_ring_close_write(r, n)) { rc = 1; break; }
      if (n < bufsz) break;   // short (possibly empty) block: end of data
    }
    fclose(f);
  } else if (!strcmp(cmd, "get")) {
    std::vector<char> hdr(4096);
    uint64_t hn = 0;
    if (dsax_ring_read_header(r, hdr.data(), hdr.size(), &hn)) return 1;
    FILE *f = fopen(argv[3], "wb");
    if (!f) return 1;
    for (;;) {
      uint64_t n = 0;
      char *b = dsax_ring_open_read(r, &n, nullptr);
      if (!b) { rc = 1; break; }
      if (n && fwrite(b, 1, n, f) != n) rc = 1;
      dsax_ring_close_read(r);
      if (n < bufsz || rc) break;
    }
    fclose(f);
  } else {
    rc = usage();
  }
  dsax_ring_disconnect(r);
  return rc;
}
