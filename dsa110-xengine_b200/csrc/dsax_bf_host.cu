// dsax_bf_host.cu -- beamformer entry points of the C-ABI and the host-side
// conversion of FP64 weights to the BF16 UMMA operand image.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"

using namespace dsax;

namespace {

// Round-to-nearest-even FP32 -> BF16 (keep the upper 16 bits, adding half an
// ulp of the kept part plus the tie-breaking lsb); NaN stays a quiet NaN.
uint16_t f32_to_bf16_rne(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0;
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// Byte offset of 16-byte chunk `chunk` of row `row` in a K-major 128-byte
// swizzled tile (8-row x 128-byte atoms), as the kernels write it.
uint32_t sw128_off(uint32_t row, uint32_t chunk) {
  return (row >> 3) * 1024u + (row & 7u) * 128u + (((chunk ^ (row & 7u)) & 7u) << 4);
}

constexpr size_t kWTile = 16384;  // 128 rows x 128 B
constexpr size_t kWPerGB = 4 * kWTile;  // [2 pol][2 kb] per (group, beam tile)
constexpr size_t kWPerGB8 = 2 * kWTile;  // FP8: [2 pol][1 kb] per (group, beam tile)

// FP32 -> E4M3 (1 sign, 4 exponent bits with bias 7, 3 mantissa bits; no
// infinities, 0x7F/0xFF are NaN), round to nearest even, saturating at 448.
uint8_t f32_to_e4m3_rne(float f) {
  const uint8_t sign = std::signbit(f) ? 0x80 : 0x00;
  double a = std::fabs((double)f);
  if (std::isnan(f)) return 0x7F;
  if (a == 0.0) return sign;
  if (a >= 448.0) return sign | 0x7E;
  int e = (int)std::floor(std::log2(a));
  if (e < -6) {   // subnormal: units of 2^-9
    const double m = std::nearbyint(std::ldexp(a, 9));
    return sign | (uint8_t)m;   // m == 8 is the smallest normal, 0x08
  }
  if (std::ldexp(1.0, e) > a) --e;          // guard against log2 rounding
  if (std::ldexp(1.0, e + 1) <= a) ++e;
  double m = std::nearbyint((a / std::ldexp(1.0, e) - 1.0) * 8.0);
  if (m >= 8.0) {
    m = 0.0;
    ++e;
  }
  if (e > 8 || (e == 8 && m > 6.0)) return sign | 0x7E;
  return sign | (uint8_t)(((e + 7) << 3) | (int)m);
}

}  // namespace

extern "C" {

int dsax_set_weights(dsax_ctx *c, const double *wre, const double *wim) {
  if (!c || !wre || !wim) return DSAX_ERR_ARG;
  const int ngrp = c->cfg.nchan / 8, nbeam = c->cfg.nbeam;
  if (c->cfg.nchan % 8 || nbeam < 64 || nbeam % 64)
    return set_error(c, DSAX_ERR_ARG, "beamformer needs nchan %% 8 == 0 and nbeam %% 64 == 0");
  const int nbt = nbeam / 64;
  const size_t nbytes = (size_t)ngrp * nbt * kWPerGB;
  std::vector<uint8_t> img(nbytes, 0);
  for (int g = 0; g < ngrp; ++g)
    for (int bt = 0; bt < nbt; ++bt)
      for (int pol = 0; pol < 2; ++pol)
        for (int kb = 0; kb < 2; ++kb)
          for (int m = 0; m < 128; ++m)
            for (int j = 0; j < 8; ++j)
              for (int i = 0; i < 4; ++i) {
                const int ant = 32 * kb + 4 * j + i;
                const int beam = 64 * bt + (m & 63);
                const size_t wi_ = (((size_t)g * 2 + pol) * nbeam + beam) * 64 + ant;
                const double wr = wre[wi_], wi = wim[wi_];
                const double c0 = m < 64 ? wr : wi;     // multiplies x_re
                const double c1 = m < 64 ? -wi : wr;    // multiplies x_im
                const size_t off = (((size_t)(g * nbt + bt) * 2 + pol) * 2 + kb) * kWTile +
                                   sw128_off((uint32_t)m, (uint32_t)j) + 4 * i;
                const uint16_t b0 = f32_to_bf16_rne((float)c0), b1 = f32_to_bf16_rne((float)c1);
                memcpy(&img[off], &b0, 2);
                memcpy(&img[off + 2], &b1, 2);
              }
  DeviceGuard dg(c->device);
  int rc = ensure_buffer(c, c->aux[AUX_WIMG_BF16], nbytes, "beamformer weights");
  if (rc != DSAX_OK) return rc;
  cudaError_t e = cudaMemcpyAsync(c->aux[AUX_WIMG_BF16].ptr, img.data(), nbytes,
                                  cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "upload weights");
  // FP8 E4M3 image with a per-antenna power-of-two scale.  Antenna a's
  // ideal exponent e_a puts its largest |coefficient| times 2^e_a in
  // [128, 256) (E4M3 tops out at 448).  The data of antenna a are scaled by
  // 2^d_a (an exponent shift in the kernel, exact for 4-bit integers while
  // d_a is in [-6, 5]) and its weights stored as q = e4m3(2^(E - d_a) w), so
  // every product carries the common factor 2^E, which the epilogue removes
  // from the power (2^-2E).  E = max(min e, max e - 6), at most min e + 5,
  // keeps d_a = E - e_a in range for spreads up to 11 octaves; beyond that
  // the antennas with the smallest weights are clamped (scaled by less than
  // their ideal 2^e_a, so they lose precision but never saturate).  Equal
  // exponents (for instance unit-magnitude weights) need no shift at all.
  {
    int ea[64];
    bool live[64];
    int emin = 1 << 20, emax = -(1 << 20);
    for (int ant = 0; ant < 64; ++ant) {
      double mx = 0.0;
      for (int g = 0; g < ngrp; ++g)
        for (int pol = 0; pol < 2; ++pol)
          for (int b = 0; b < nbeam; ++b) {
            const size_t wi_ = (((size_t)g * 2 + pol) * nbeam + b) * 64 + ant;
            mx = std::max(mx, std::max(std::fabs(wre[wi_]), std::fabs(wim[wi_])));
          }
      live[ant] = mx > 0.0;
      ea[ant] = live[ant] ? std::min(50, std::max(-50, 7 - (int)std::floor(std::log2(mx)))) : 0;
      if (live[ant]) {
        emin = std::min(emin, ea[ant]);
        emax = std::max(emax, ea[ant]);
      }
    }
    const int E = emin <= emax ? std::min(emin + 5, std::max(emin, emax - 6)) : 0;
    int d[64];
    signed char add[64];
    bool any = false;
    for (int ant = 0; ant < 64; ++ant) {
      d[ant] = live[ant] ? std::min(5, std::max(-6, E - ea[ant])) : 0;
      add[ant] = (signed char)(d[ant] * 8);
      any |= d[ant] != 0;
    }
    const size_t nb8 = (size_t)ngrp * nbt * kWPerGB8;
    std::vector<uint8_t> img8(nb8, 0);
    for (int g = 0; g < ngrp; ++g)
      for (int bt = 0; bt < nbt; ++bt)
        for (int pol = 0; pol < 2; ++pol)
          for (int m = 0; m < 128; ++m)
            for (int ant = 0; ant < 64; ++ant) {
              const int beam = 64 * bt + (m & 63);
              const size_t wi_ = (((size_t)g * 2 + pol) * nbeam + beam) * 64 + ant;
              const double wr = wre[wi_], wi = wim[wi_];
              const double sc = std::ldexp(1.0, E - d[ant]);
              const double c0 = (m < 64 ? wr : wi) * sc, c1 = (m < 64 ? -wi : wr) * sc;
              const size_t off = (((size_t)(g * nbt + bt) * 2 + pol)) * kWTile +
                                 sw128_off((uint32_t)m, (uint32_t)(ant / 8)) + 2 * (ant % 8);
              img8[off] = f32_to_e4m3_rne((float)c0);
              img8[off + 1] = f32_to_e4m3_rne((float)c1);
            }
    if ((rc = ensure_buffer(c, c->aux[AUX_WIMG_FP8], nb8 + 256, "FP8 beamformer weights")) != DSAX_OK)
      return rc;
    uint8_t *d8 = static_cast<uint8_t *>(c->aux[AUX_WIMG_FP8].ptr);
    e = cudaMemcpyAsync(d8, img8.data(), nb8, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d8 + nb8, add, 64, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_check(c, e, "upload FP8 weights");
    c->fp8_pscale = (float)std::ldexp(1.0, -2 * E);
    c->fp8_shift = any ? 1 : 0;
    c->fp8_img_bytes = nb8;
  }
  c->weights_ready = 1;
  c->weights_nchan = c->cfg.nchan;
  return DSAX_OK;
}

// Geometric (fan-beam) weights in FP64, restating calc_weights
// (src/dsaX_beamformer.cu:421-449) with the calibration normalisation of
// init_weights (:559-602): for channel group g (centre frequency
// fch1 - (8g + 4) x 250/8192 MHz), pol p, beam b (offset theta_b =
// sep x (127 - b) arcmin) and antenna a (easting pos_a),
//   w = exp(i afac pos_a) x cal / |cal|^2,  afac = -2 pi nu theta_b / c,
// zero for flagged antennas; then the BF16 operand image as dsax_set_weights.
int dsax_set_geometric_weights(dsax_ctx *c, const double *antpos, const double *cal,
                               const int *flagged, double fch1_mhz, double sep_arcmin) {
  if (!c || !antpos || !cal) return DSAX_ERR_ARG;
  const int ngrp = c->cfg.nchan / 8, nbeam = c->cfg.nbeam;
  if (c->cfg.nchan % 8 || nbeam < 64 || nbeam % 64)
    return set_error(c, DSAX_ERR_ARG, "beamformer needs nchan %% 8 == 0 and nbeam %% 64 == 0");
  const double kPi = 3.14159265358979323846, kC = 299792458.0;
  std::vector<double> wre((size_t)ngrp * 2 * nbeam * 64), wim(wre.size());
  for (int g = 0; g < ngrp; ++g)
    for (int pol = 0; pol < 2; ++pol)
      for (int b = 0; b < nbeam; ++b)
        for (int a = 0; a < 64; ++a) {
          const double *cc = cal + (((size_t)a * ngrp + g) * 2 + pol) * 2;
          double cr = cc[0], ci = cc[1];
          const double n2 = cr * cr + ci * ci;
          if (n2 != 0.0) { cr /= n2; ci /= n2; }
          if (flagged && flagged[a]) { cr = 0.0; ci = 0.0; }
          const double nu = (fch1_mhz - (8.0 * g + 4.0) * 250.0 / 8192.0) * 1e6;
          const double theta = sep_arcmin * (127.0 - b) * kPi / 10800.0;
          const double ph = -2.0 * kPi * nu * theta / kC * antpos[a];
          const double tr = cos(ph), ti = sin(ph);
          const size_t o = (((size_t)g * 2 + pol) * nbeam + b) * 64 + a;
          wre[o] = tr * cr - ti * ci;
          wim[o] = ti * cr + tr * ci;
        }
  return dsax_set_weights(c, wre.data(), wim.data());
}

int dsax_set_two_arm_weights(dsax_ctx *c, const double *antpos_e, const double *antpos_n,
                             const int *arm, const double *cal, const int *flagged,
                             double sfreq_mhz, double sep_arcmin, double dec_deg) {
  if (!c || !antpos_e || !antpos_n || !arm || !cal) return DSAX_ERR_ARG;
  const int ngrp = c->cfg.nchan / 8, nbeam = c->cfg.nbeam, nb_arm = nbeam / 2;
  if (c->cfg.nchan % 8 || nbeam < 128 || nbeam % 128)
    return set_error(c, DSAX_ERR_ARG, "two-arm weights need nchan %% 8 == 0, nbeam %% 128 == 0");
  for (int a = 0; a < 64; ++a)
    if (arm[a] != 0 && arm[a] != 1 && arm[a] != -1)
      return set_error(c, DSAX_ERR_ARG, "arm[%d] must be 0 (E-W), 1 (N-S) or -1 (unused)", a);
  const double kPi = 3.14159265358979323846, kC = 299792458.0;
  std::vector<double> wre((size_t)ngrp * 2 * nbeam * 64, 0.0), wim(wre.size(), 0.0);
  for (int g = 0; g < ngrp; ++g) {
    const double nu = (sfreq_mhz - g * 250.0 / 1024.0) * 1e6;   // :1131
    for (int pol = 0; pol < 2; ++pol)
      for (int b = 0; b < nbeam; ++b) {
        const int A = b / nb_arm, bb = b - A * nb_arm;
        double theta = sep_arcmin * ((nb_arm / 2 - 1) - bb) * kPi / 10800.0;
        if (A == 1) theta -= dec_deg * kPi / 180.0;
        const double afac = -2.0 * kPi * nu * theta / kC;
        for (int a = 0; a < 64; ++a) {
          if (arm[a] != A || (flagged && flagged[a])) continue;
          const double *cc = cal + (((size_t)a * ngrp + g) * 2 + pol) * 2;
          double cr = cc[0], ci = cc[1];
          const double n = std::sqrt(cr * cr + ci * ci);   // unit gain phase (:891-895)
          if (n != 0.0) { cr /= n; ci /= n; }
          const double ph = afac * (A == 0 ? antpos_e[a] : antpos_n[a]);
          const double tr = std::cos(ph), ti = std::sin(ph);
          const size_t o = (((size_t)g * 2 + pol) * nbeam + b) * 64 + a;
          wre[o] = tr * cr - ti * ci;
          wim[o] = ti * cr + tr * ci;
        }
      }
  }
  return dsax_set_weights(c, wre.data(), wim.data());
}

int dsax_beamform(dsax_ctx *c, const void *blk, void *out_u8, void *out_f32, int mem) {
  if (!c || !blk || (!out_u8 && !out_f32)) return DSAX_ERR_ARG;
  if (!c->weights_ready) return set_error(c, DSAX_ERR_ARG, "dsax_set_weights not called");
  const dsax_config &cf = c->cfg;
  const int ppo = cf.bf_pkt_per_out;
  if (cf.nchan % 8 || cf.nbeam % 64 || cf.npkt % 16 || ppo <= 0 || cf.npkt % ppo ||
      !(ppo == 4 || ppo == 8 || ppo % 16 == 0))
    return set_error(c, DSAX_ERR_ARG,
                     "beamformer needs nchan%%8==0, nbeam%%64==0, npkt%%16==0, npkt%%ppo==0, "
                     "ppo in {4, 8, 16k}");
  if (mem != DSAX_MEM_HOST && mem != DSAX_MEM_DEVICE) return DSAX_ERR_ARG;
  DeviceGuard dg(c->device);
  const size_t nin = dsax_block_bytes(&cf, DSAX_FMT_CAPTURED);
  const size_t nout = dsax_beam_bytes(&cf);
  BfArgs a{};
  a.wimg = static_cast<const uint8_t *>(c->aux[AUX_WIMG_BF16].ptr);
  a.err = c->d_err;
  a.npkt = cf.npkt;
  a.nant_in = cf.nant_in;
  a.nchan = cf.nchan;
  a.nbeam = cf.nbeam;
  a.ppo = ppo;
  a.scale = cf.bf_scale;
  a.wait_limit_ns = cf.wait_limit_ns;
  a.pscale = 1.0f;
  a.path = cf.bf_path;
  a.variant = cf.bf_variant;
  if (cf.bf_fp8) {   // E4M3 operands, per-antenna data exponents, power by 2^-2E
    a.fp8 = 1;
    a.wimg = static_cast<const uint8_t *>(c->aux[AUX_WIMG_FP8].ptr);
    a.pscale = c->fp8_pscale;
    a.e4m3_add = c->fp8_shift
                     ? reinterpret_cast<const signed char *>(a.wimg + c->fp8_img_bytes)
                     : nullptr;
  }
  if (c->agc_on) {   // per-beam scale from the previous blocks; this block's power for the next
    a.agc_scale = agc_scale_ptr(c->aux[AUX_AGC].ptr, cf.nbeam);
    a.beam_power = agc_power_ptr(c->aux[AUX_AGC].ptr, cf.nbeam);
  }
  auto agc_after = [&]() -> bool {
    return !c->agc_on ||
           launch_agc_update(c->aux[AUX_AGC].ptr, cf.nbeam, cf.nchan / 8, cf.npkt / 16, c->stream) == 0;
  };
  if (mem == DSAX_MEM_DEVICE) {
    if (!aligned16(blk)) return set_error(c, DSAX_ERR_ARG, "block must be 16-byte aligned");
    a.in = static_cast<const uint8_t *>(blk);
    a.out_u8 = static_cast<uint8_t *>(out_u8);
    a.out_f32 = static_cast<float *>(out_f32);
    if (launch_beamform(a, c->num_sms, c->stream) != 0 || !agc_after())
      return cuda_check(c, cudaGetLastError(), "beamformer launch");
    return DSAX_OK;
  }
  int rc;
  if ((rc = ensure_buffer(c, c->in_buf, nin, "input block")) != DSAX_OK) return rc;
  if (out_u8 && (rc = ensure_buffer(c, c->aux[AUX_BEAM_U8], nout, "beams")) != DSAX_OK) return rc;
  if (out_f32 && (rc = ensure_buffer(c, c->aux[AUX_BEAM_F32], nout * 4, "beam power")) != DSAX_OK)
    return rc;
  cudaError_t e = cudaMemcpyAsync(c->in_buf.ptr, blk, nin, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_check(c, e, "H2D block");
  a.in = static_cast<const uint8_t *>(c->in_buf.ptr);
  a.out_u8 = out_u8 ? static_cast<uint8_t *>(c->aux[AUX_BEAM_U8].ptr) : nullptr;
  a.out_f32 = out_f32 ? static_cast<float *>(c->aux[AUX_BEAM_F32].ptr) : nullptr;
  if (launch_beamform(a, c->num_sms, c->stream) != 0 || !agc_after())
    return cuda_check(c, cudaGetLastError(), "beamformer launch");
  if (out_u8 && (e = cudaMemcpyAsync(out_u8, a.out_u8, nout, cudaMemcpyDeviceToHost, c->stream)) !=
                    cudaSuccess)
    return cuda_check(c, e, "D2H beams");
  if (out_f32 && (e = cudaMemcpyAsync(out_f32, a.out_f32, nout * 4, cudaMemcpyDeviceToHost,
                                      c->stream)) != cudaSuccess)
    return cuda_check(c, e, "D2H beam power");
  return dsax_sync(c);
}

}  // extern "C"
