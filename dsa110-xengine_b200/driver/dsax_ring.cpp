// dsax_ring.cpp -- POSIX shared-memory block ring (see dsax_ring.h).
#include "dsax_ring.h"

#include <errno.h>
#include <fcntl.h>
#include <pthread.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include <cstdio>
#include <new>

namespace {

constexpr uint64_t kMagic = 0x44534158524e4731ull;   // "DSAXRNG1"
constexpr uint64_t kAlign = 4096;
constexpr uint64_t kMaxBufs = 1024;

struct Shared {
  uint64_t magic, nbufs, bufsz, hdrsz;
  uint64_t data_off, total;
  pthread_mutex_t mu;
  pthread_cond_t cv;
  uint64_t wcount, rcount;     // blocks written / read so far
  uint64_t hdr_bytes;
  int hdr_filled, hdr_read;
  uint64_t bytes[kMaxBufs];    // valid bytes of each block slot
};

uint64_t up(uint64_t n) { return (n + kAlign - 1) & ~(kAlign - 1); }

void deadline(timespec *ts, double s) {
  clock_gettime(CLOCK_REALTIME, ts);
  const long ns = (long)((s - (double)(long)s) * 1e9);
  ts->tv_sec += (time_t)s + (ts->tv_nsec + ns) / 1000000000L;
  ts->tv_nsec = (ts->tv_nsec + ns) % 1000000000L;
}

}  // namespace

struct dsax_ring {
  Shared *s;
  size_t map_bytes;
  double timeout;
  bool reading, writing;
};

// Waits (bounded) until pred() holds; called with the mutex held.
template <class P>
static int wait_for(dsax_ring *r, P pred) {
  timespec ts;
  deadline(&ts, r->timeout);
  while (!pred()) {
    const int e = pthread_cond_timedwait(&r->s->cv, &r->s->mu, &ts);
    if (e == ETIMEDOUT && !pred()) return -1;
  }
  return 0;
}

extern "C" {

int dsax_ring_create(const char *name, uint64_t nbufs, uint64_t bufsz, uint64_t hdrsz) {
  if (!name || nbufs < 1 || nbufs > kMaxBufs || bufsz < 1) return -1;
  const uint64_t data_off = up(sizeof(Shared) + hdrsz);
  const uint64_t total = data_off + nbufs * up(bufsz);
  int fd = shm_open(name, O_CREAT | O_EXCL | O_RDWR, 0600);
  if (fd < 0) return -2;
  if (ftruncate(fd, (off_t)total) != 0) {
    close(fd);
    shm_unlink(name);
    return -3;
  }
  void *p = mmap(nullptr, total, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (p == MAP_FAILED) {
    shm_unlink(name);
    return -4;
  }
  Shared *s = static_cast<Shared *>(p);
  memset(s, 0, sizeof(Shared));
  pthread_mutexattr_t ma;
  pthread_mutexattr_init(&ma);
  pthread_mutexattr_setpshared(&ma, PTHREAD_PROCESS_SHARED);
  pthread_mutex_init(&s->mu, &ma);
  pthread_condattr_t ca;
  pthread_condattr_init(&ca);
  pthread_condattr_setpshared(&ca, PTHREAD_PROCESS_SHARED);
  pthread_cond_init(&s->cv, &ca);
  s->nbufs = nbufs;
  s->bufsz = bufsz;
  s->hdrsz = hdrsz;
  s->data_off = data_off;
  s->total = total;
  __sync_synchronize();
  s->magic = kMagic;
  munmap(p, total);
  return 0;
}

int dsax_ring_destroy(const char *name) { return name && shm_unlink(name) == 0 ? 0 : -1; }

dsax_ring *dsax_ring_connect(const char *name, double timeout_s) {
  if (!name) return nullptr;
  int fd = shm_open(name, O_RDWR, 0600);
  if (fd < 0) return nullptr;
  struct stat st;
  if (fstat(fd, &st) != 0 || (uint64_t)st.st_size < sizeof(Shared)) {
    close(fd);
    return nullptr;
  }
  void *p = mmap(nullptr, (size_t)st.st_size, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (p == MAP_FAILED) return nullptr;
  Shared *s = static_cast<Shared *>(p);
  if (s->magic != kMagic || s->total != (uint64_t)st.st_size) {
    munmap(p, (size_t)st.st_size);
    return nullptr;
  }
  dsax_ring *r = new (std::nothrow) dsax_ring{s, (size_t)st.st_size, timeout_s > 0 ? timeout_s : 60.0,
                                              false, false};
  if (!r) munmap(p, (size_t)st.st_size);
  return r;
}

void dsax_ring_disconnect(dsax_ring *r) {
  if (!r) return;
  munmap(r->s, r->map_bytes);
  delete r;
}

uint64_t dsax_ring_bufsz(const dsax_ring *r) { return r ? r->s->bufsz : 0; }
uint64_t dsax_ring_nbufs(const dsax_ring *r) { return r ? r->s->nbufs : 0; }

char *dsax_ring_data(dsax_ring *r, uint64_t *total_bytes) {
  if (!r) return nullptr;
  if (total_bytes) *total_bytes = r->s->nbufs * up(r->s->bufsz);
  return reinterpret_cast<char *>(r->s) + r->s->data_off;
}

int dsax_ring_write_header(dsax_ring *r, const char *hdr, uint64_t n) {
  if (!r || !hdr || n > r->s->hdrsz) return -1;
  Shared *s = r->s;
  pthread_mutex_lock(&s->mu);
  memcpy(reinterpret_cast<char *>(s) + sizeof(Shared), hdr, n);
  s->hdr_bytes = n;
  s->hdr_filled = 1;
  pthread_cond_broadcast(&s->cv);
  pthread_mutex_unlock(&s->mu);
  return 0;
}

int dsax_ring_read_header(dsax_ring *r, char *hdr, uint64_t cap, uint64_t *n) {
  if (!r || !hdr) return -1;
  Shared *s = r->s;
  pthread_mutex_lock(&s->mu);
  int rc = wait_for(r, [&] { return s->hdr_filled != 0; });
  if (rc == 0) {
    const uint64_t m = s->hdr_bytes < cap ? s->hdr_bytes : cap;
    memcpy(hdr, reinterpret_cast<char *>(s) + sizeof(Shared), m);
    if (n) *n = m;
    s->hdr_read = 1;
  }
  pthread_mutex_unlock(&s->mu);
  return rc;
}

char *dsax_ring_open_write(dsax_ring *r, uint64_t *block_id) {
  if (!r || r->writing) return nullptr;
  Shared *s = r->s;
  pthread_mutex_lock(&s->mu);
  int rc = wait_for(r, [&] { return s->wcount - s->rcount < s->nbufs; });
  const uint64_t slot = s->wcount % s->nbufs;
  if (block_id) *block_id = s->wcount;
  pthread_mutex_unlock(&s->mu);
  if (rc != 0) return nullptr;
  r->writing = true;
  return reinterpret_cast<char *>(s) + s->data_off + slot * up(s->bufsz);
}

int dsax_ring_close_write(dsax_ring *r, uint64_t bytes) {
  if (!r || !r->writing || bytes > r->s->bufsz) return -1;
  Shared *s = r->s;
  pthread_mutex_lock(&s->mu);
  s->bytes[s->wcount % s->nbufs] = bytes;
  __sync_synchronize();
  s->wcount++;
  pthread_cond_broadcast(&s->cv);
  pthread_mutex_unlock(&s->mu);
  r->writing = false;
  return 0;
}

char *dsax_ring_open_read(dsax_ring *r, uint64_t *bytes, uint64_t *block_id) {
  if (!r || r->reading) return nullptr;
  Shared *s = r->s;
  pthread_mutex_lock(&s->mu);
  int rc = wait_for(r, [&] { return s->wcount > s->rcount; });
  const uint64_t slot = s->rcount % s->nbufs;
  if (bytes) *bytes = rc == 0 ? s->bytes[slot] : 0;
  if (block_id) *block_id = s->rcount;
  pthread_mutex_unlock(&s->mu);
  if (rc != 0) return nullptr;
  r->reading = true;
  return reinterpret_cast<char *>(s) + s->data_off + slot * up(s->bufsz);
}

int dsax_ring_close_read(dsax_ring *r) {
  if (!r || !r->reading) return -1;
  Shared *s = r->s;
  pthread_mutex_lock(&s->mu);
  s->rcount++;
  pthread_cond_broadcast(&s->cv);
  pthread_mutex_unlock(&s->mu);
  r->reading = false;
  return 0;
}

}  // extern "C"
