/* ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of astroflow's dedispersion hot path (see dd_oracle.h for the
 * role and the parity pin).  Arithmetic is strict IEEE (built with
 * -ffp-contract=off and no fast-math); where the reference's result depends on
 * its compiler flags (fused multiply-add, reciprocal-multiply), a `variant` bit
 * selects the form, and the tests pin which form matches the reference's own
 * build.  The fast-math single-precision reciprocal and division that the
 * reference's device code uses for its subband delay tables are not
 * reproduced here: orc_subband_tables_ieee is the IEEE statement of the same
 * formulas, and the sums (orc_subband_sums) take the tables as an input so
 * that the exact device tables can be fed in.
 */
#include "dd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define KDM 4148.808f /* dedispered.cu:332, cpucal.hpp:128 */

static inline uint64_t ld(const void* p, int nbits, size_t i) {
  switch (nbits) {
    case 8: return ((const uint8_t*)p)[i];
    case 16: return ((const uint16_t*)p)[i];
    default: return ((const uint32_t*)p)[i];
  }
}
static inline void st(void* p, int nbits, size_t i, uint64_t v) {
  switch (nbits) {
    case 8: ((uint8_t*)p)[i] = (uint8_t)v; break;
    case 16: ((uint16_t*)p)[i] = (uint16_t)v; break;
    default: ((uint32_t*)p)[i] = (uint32_t)v; break;
  }
}
static inline uint64_t vmax_of(int nbits) {
  return nbits == 8 ? 255u : nbits == 16 ? 65535u : 4294967295u;
}

/* dedispered.cu:1003-1005: h_freq[i] = header.fch1 + i*header.foff, evaluated in
 * float (Header's fields are float, data.h:24-31) and stored as double. */
void orc_freq_table_header(float fch1, float foff, int nchans, double* freq) {
  /* the reference build (-ffast-math, FMA) contracts fch1 + i*foff into one fmaf */
  for (int i = 0; i < nchans; ++i) freq[i] = (double)fmaf((float)(size_t)i, foff, fch1);
}

/* src/data/filterbank.cpp:445-449: frequency_table[i] = fch1 + i*foff in double. */
void orc_freq_table_fil(double fch1, double foff, int nchans, double* freq) {
  /* contracted into fma by the reference build (-Ofast with FMA) */
  for (int i = 0; i < nchans; ++i) freq[i] = fma((double)i, foff, fch1);
}

/* dedispered.cu:1007-1027 (also cpucal.hpp:85-110 and dedispered.cu:529-548):
 * the band edges are read back as float, the channel index is the truncated
 * float expression (f - fmin)/(fmax - fmin)*(nchans-1).  Returns 1 when the
 * range is outside the band (the reference throws std::invalid_argument). */
int orc_chan_range(const double* freq, int nchans, float freq_start, float freq_end,
                   long* chan_start, long* chan_end) {
  float fmin = (float)freq[0];
  float fmax = (float)freq[nchans - 1];
  if (freq_start < fmin || freq_end > fmax) return 1;
  float n1 = (float)(size_t)(nchans - 1);
  float span = fmax - fmin;
  float a = (freq_start - fmin) / span;
  float b = (freq_end - fmin) / span;
  size_t cs = (size_t)(a * n1);
  size_t ce = (size_t)(b * n1);
  if (ce > (size_t)(nchans - 1)) ce = (size_t)(nchans - 1);
  *chan_start = (long)cs;
  *chan_end = (long)ce;
  if (cs >= (size_t)nchans || ce >= (size_t)nchans) return 2;
  return 0;
}

/* dedispered.cu:1029, cpucal.hpp:115: (size_t)((dm_high - dm_low)/dm_step) + 1 in float. */
long orc_dm_steps(float dm_low, float dm_high, float dm_step) {
  float q = (dm_high - dm_low) / dm_step;
  return (long)(size_t)q + 1;
}

static inline float dm_at(float lo, float idx, float step, int variant) {
  if (variant & ORC_FMA_DM) return fmaf(idx, step, lo);
  float p = idx * step;
  return lo + p;
}

/* IEEE statement of the subband tables:
 *  - coarse delays, pre_calculate_dedispersion_kernel (dedispered.cu:318-335)
 *    launched at dedispered.cu:1129-1141 for the nominal DMs
 *    dm_j = dm_low + j*(ndm0*dm_step), followed by the integer division by the
 *    downsample factor (divide_delay_inplace_kernel, dedispered.cu:379-382);
 *    a nominal DM whose value exceeds dm_high_coarse is skipped by the kernel
 *    and its row keeps the (zero-filled) allocation contents;
 *  - residual shifts, compute_residual2_kernel (dedispered.cu:385-413) at the
 *    subband centre frequency freq[(ch0+ch1-1)/2] (dedispered.cu:1151-1157).
 * delay1 is [ceil(dm_steps/ndm0)][chan_end-chan_start+1]; residual2 is
 * [dm_steps][nsb]. */
void orc_subband_tables_ieee(const double* freq, long chan_start, long chan_end, float dm_low,
                             float dm_step, long dm_steps, int sb_width, int ndm0, double tsamp,
                             int ds, int variant, int* delay1, int* residual2) {
  const long dch = chan_end - chan_start + 1;
  const long nsb = (dch + sb_width - 1) / sb_width;
  const long ndm_nom = (dm_steps + ndm0 - 1) / ndm0;
  const float ref = (float)freq[chan_end];
  const float ref2 = ref * ref;
  const float step_c = dm_step * (float)ndm0;
  const float high_c = dm_low + (float)(size_t)(ndm_nom - 1) * step_c;
  for (long j = 0; j < ndm_nom; ++j) {
    float dm = dm_at(dm_low, (float)(unsigned)j, step_c, variant);
    for (long c = 0; c < dch; ++c) {
      int v = 0;
      if (!(dm > high_c)) {
        double f = freq[chan_start + c];
        float f2 = (float)(f * f);
        float delay = KDM * dm * (1.0f / f2 - 1.0f / ref2);
        v = (int)roundf((float)((double)delay / tsamp));
      }
      delay1[j * dch + c] = v / ds;
    }
  }
  const float tbin = (float)(tsamp * ds);
  for (long m = 0; m < dm_steps; ++m) {
    long j = m / ndm0;
    float dmj = dm_at(dm_low, (float)(size_t)(j * ndm0), dm_step, variant);
    float dmm = dm_at(dm_low, (float)(size_t)m, dm_step, variant);
    float dmd = dmm - dmj;
    for (long sb = 0; sb < nsb; ++sb) {
      long ch0 = chan_start + sb * sb_width;
      long ch1 = ch0 + sb_width < chan_end + 1 ? ch0 + sb_width : chan_end + 1;
      double f = freq[(ch0 + ch1 - 1) / 2];
      float f2 = (float)(f * f);
      float delay = KDM * dmd * (1.0f / f2 - 1.0f / ref2);
      float bins_f = delay / tbin;
      residual2[m * nsb + sb] = (int)floorf(bins_f + 0.5f);
    }
  }
}

/* Exact-physics table in FP64 for comparison: round(K*DM*(f^-2 - fref^-2)/tsamp)/ds,
 * with the reference's DM grid and reference channel (the top channel). */
void orc_delay_table_fp64(const double* freq, long chan_start, long chan_end, float dm_low,
                          float dm_step, long ndm, double tsamp, int ds, int* delay) {
  const long dch = chan_end - chan_start + 1;
  const double ref = freq[chan_end];
  for (long m = 0; m < ndm; ++m) {
    double dm = (double)dm_low + (double)m * (double)dm_step;
    for (long c = 0; c < dch; ++c) {
      double f = freq[chan_start + c];
      double d = 4148.808 * dm * (1.0 / (f * f) - 1.0 / (ref * ref)) / tsamp;
      delay[m * dch + c] = (int)floor(d + 0.5) / ds;
    }
  }
}

/* Per-DM channel delays of the CPU brute force, cpucal.hpp:119-132:
 * float freq = frequency_table[ch]; float delay = 4148.808f*dm*(1/f^2 - 1/ref^2);
 * delay index = (int)round(delay / tsamp) with tsamp in double.  The table holds
 * the channels [chan_start, chan_end) (the top channel is not summed). */
void orc_cpu_delay_table(const double* freq, long chan_start, long chan_end, float dm_low,
                         float dm_step, long dm_steps, double tsamp, int variant, int* delay) {
  const long nc = chan_end - chan_start;
  const float ref = (float)freq[chan_end];
  const float inv_ref2 = 1.0f / (ref * ref);
  const double inv_tsamp = 1.0 / tsamp;
  for (long s = 0; s < dm_steps; ++s) {
    float dm = dm_at(dm_low, (float)(size_t)s, dm_step, variant);
    float kd = KDM * dm;
    float kb = kd * inv_ref2;
    for (long c = 0; c < nc; ++c) {
      float fr = (float)freq[chan_start + c];
      float a = 1.0f / (fr * fr);
      float d;
      if (variant & ORC_CPU_EXPFMA) d = fmaf(kd, a, -kb);
      else if (variant & ORC_CPU_EXPAND) { float ka = kd * a; d = ka - kb; }
      else d = kd * (a - inv_ref2);
      double q = (variant & ORC_RECIP_TSAMP) ? (double)d * inv_tsamp : (double)d / tsamp;
      delay[s * nc + c] = (int)round(q);
    }
  }
}

/* cpucal::dedispered_fil_omp (cpucal.hpp:75-201), raw sums before the image step:
 * slices of round(t_sample/tsamp) input samples; in slice s the output column ti
 * sums data[(start + ti*ds + delay[ch]) * nchans + ch] over ch in
 * [chan_start, chan_end) for the terms with start + ti*ds + delay < ndata.
 * Output: the slices' [ndm][cols_s] uint64 arrays back to back.  delay_in, when
 * not NULL, replaces the computed [ndm][chan_end-chan_start] delay table. */
int orc_bruteforce_cpu(const void* data, int nbits, long ndata, int nchans, const double* freq,
                       double tsamp, float dm_low, float dm_high, float freq_start,
                       float freq_end, float dm_step, int ds, float t_sample, int variant,
                       const int* delay_in, uint64_t* out, long out_cap, long* nslices,
                       long* slice_cols, long slice_cap, long* ndm) {
  long cs, ce;
  if (orc_chan_range(freq, nchans, freq_start, freq_end, &cs, &ce)) return 1;
  if (cs >= ce) return 1;
  if (ds < 1) return 1;
  if (dm_low > dm_high || dm_low < 0 || dm_step <= 0) return 1;
  if (t_sample > (double)ndata * tsamp) return 1;
  const long steps = orc_dm_steps(dm_low, dm_high, dm_step);
  const long nc = ce - cs;
  int* delay = (int*)malloc(sizeof(int) * (size_t)(steps * nc));
  if (!delay) return 9;
  if (delay_in)
    memcpy(delay, delay_in, sizeof(int) * (size_t)(steps * nc));
  else
    orc_cpu_delay_table(freq, cs, ce, dm_low, dm_step, steps, tsamp, variant, delay);
  const size_t sps = (size_t)round((double)t_sample / tsamp);
  const size_t total = ((size_t)ndata + sps - 1) / sps;
  if ((long)total > slice_cap) { free(delay); return 3; }
  size_t off = 0;
  for (size_t s = 0; s < total; ++s) {
    size_t start = s * sps;
    size_t end = start + sps < (size_t)ndata ? start + sps : (size_t)ndata;
    size_t cols = (end - start + ds - 1) / ds;
    if ((long)(off + steps * cols) > out_cap) { free(delay); return 4; }
    for (long m = 0; m < steps; ++m) {
      const int* dl = delay + m * nc;
      for (size_t ti = 0; ti < cols; ++ti) {
        size_t base = start + ti * ds;
        uint64_t sum = 0;
        for (long c = 0; c < nc; ++c) {
          size_t idx = base + (size_t)(long)dl[c];
          if (idx < (size_t)ndata) sum += ld(data, nbits, idx * nchans + cs + c);
        }
        out[off + m * cols + ti] = sum;
      }
    }
    off += steps * cols;
    slice_cols[s] = (long)cols;
  }
  *nslices = (long)total;
  *ndm = steps;
  free(delay);
  return 0;
}

/* Two-stage subband sums of the reference GPU path (dedispered.cu:416-476,
 * 1196-1235), in the time-tile-independent form
 *   inter[j][sb][u] = sum_{ch in sb} [u + d1[j][ch] < N] x[u + d1][ch]   (u < N)
 *   out[m][t]       = sum_sb [t + r2[m][sb] < N] inter[m/ndm0][sb][t + r2]
 * over the channels [chan_start, chan_end] (inclusive) of the binned input
 * (nsamp = down_ndata rows).  Output [dm_steps][nsamp] in uint64. */
int orc_subband_sums(const void* data, int nbits, long nsamp, int nchans, long chan_start,
                     long chan_end, int sb_width, int ndm0, long dm_steps, const int* delay1,
                     const int* residual2, uint64_t* out) {
  const long dch = chan_end - chan_start + 1;
  const long nsb = (dch + sb_width - 1) / sb_width;
  const long ndm_nom = (dm_steps + ndm0 - 1) / ndm0;
  uint64_t* inter = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nsb * nsamp));
  if (!inter) return 9;
  for (long j = 0; j < ndm_nom; ++j) {
    const int* d1 = delay1 + j * dch;
    for (long sb = 0; sb < nsb; ++sb) {
      long c0 = sb * sb_width;
      long c1 = c0 + sb_width < dch ? c0 + sb_width : dch;
      uint64_t* row = inter + sb * nsamp;
      for (long u = 0; u < nsamp; ++u) {
        uint64_t s = 0;
        for (long c = c0; c < c1; ++c) {
          size_t tt = (size_t)u + (size_t)(long)d1[c];
          if (tt < (size_t)nsamp) s += ld(data, nbits, tt * nchans + chan_start + c);
        }
        row[u] = s;
      }
    }
    long m1 = (j + 1) * ndm0 < dm_steps ? (j + 1) * ndm0 : dm_steps;
    for (long m = j * ndm0; m < m1; ++m) {
      const int* r2 = residual2 + m * nsb;
      uint64_t* o = out + m * nsamp;
      for (long t = 0; t < nsamp; ++t) o[t] = 0;
      for (long sb = 0; sb < nsb; ++sb) {
        const uint64_t* row = inter + sb * nsamp;
        size_t r = (size_t)(long)r2[sb];
        for (long t = 0; t < nsamp; ++t) {
          size_t ti = (size_t)t + r;
          if (ti < (size_t)nsamp) o[t] += row[ti];
        }
      }
    }
  }
  free(inter);
  return 0;
}

/* time_binning_kernel (dedispered.cu:337-376) with USE_SQRT_COMPRESSION:
 * v = sqrt(sum)/sqrt(vmax*cnt)*vmax in double, min(v, vmax), truncated to T. */
int orc_time_binning(const void* in, int nbits, long ndata, int nchans, int ds, void* out) {
  if (ds < 1) return 1;
  const long nout = (ndata + ds - 1) / ds;
  const uint64_t vmax = vmax_of(nbits);
  for (long k = 0; k < nout; ++k) {
    long t0 = k * ds;
    long t1 = t0 + ds < ndata ? t0 + ds : ndata;
    uint64_t cnt = (uint64_t)(t1 - t0);
    for (long c = 0; c < nchans; ++c) {
      uint64_t sum = 0;
      for (long t = t0; t < t1; ++t) sum += ld(in, nbits, (size_t)t * nchans + c);
      double s = sqrt((double)sum);
      double smax = sqrt((double)(vmax * (cnt ? cnt : 1)));
      double v = (s / (smax > 0.0 ? smax : 1.0)) * (double)vmax;
      double cl = v < (double)vmax ? v : (double)vmax;
      st(out, nbits, (size_t)k * nchans + c, (uint64_t)cl);
    }
  }
  return 0;
}

/* Window plan of iqrm_cuda::iqrm (iqrm.cu:348-397): W = floor(win_sec/tsamp)
 * samples (0 -> one window over everything), hop H = floor(hop_sec/tsamp) (0 ->
 * W), a trailing partial window when include_tail and it is longer than 4
 * samples.  The config clamps of iqrm.hpp:30-41 (win/hop >= 0) are applied. */
int orc_iqrm_windows(double win_sec, double hop_sec, int include_tail, double tsamp,
                     unsigned nsample, unsigned* t0, unsigned* t1, int cap) {
  if (win_sec < 0.0) win_sec = 0.0;
  if (hop_sec < 0.0) hop_sec = 0.0;
  unsigned W = win_sec > 0.0 ? (unsigned)floor(win_sec / tsamp) : 0u;
  unsigned H = hop_sec > 0.0 ? (unsigned)floor(hop_sec / tsamp) : W;
  int n = 0;
  if (W == 0 || W >= nsample) {
    if (n < cap) { t0[n] = 0; t1[n] = nsample; }
    return 1;
  }
  unsigned a = 0;
  while (a + W <= nsample) {
    if (n < cap) { t0[n] = a; t1[n] = a + W; }
    ++n;
    a += (H ? H : W);
  }
  if (include_tail && a < nsample) {
    if (nsample > a + 4) {
      if (n < cap) { t0[n] = a; t1[n] = nsample; }
      ++n;
    }
  }
  return n;
}

/* gen_lags_host (iqrm.cu:188-200): +-1, +-2, ..., next = max((int)(g*lag), lag+1). */
int orc_iqrm_lags(int radius, double geofactor, int* lags, int cap) {
  int n = 0;
  if (radius <= 0) return 0;
  int lag = 1;
  while (lag <= radius) {
    if (n + 1 < cap) { lags[n] = lag; lags[n + 1] = -lag; }
    n += 2;
    int nxt = (int)(geofactor * lag);
    lag = nxt > lag + 1 ? nxt : lag + 1;
  }
  return n;
}

static int cmp_float(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* Linear-interpolated percentile of the host side of run_iqrm_one_window_gpu
 * (iqrm.cu:299-306): pos in double, the difference of the two floats in float. */
static float pct(const float* v, unsigned n, float q) {
  if (n == 1) return v[0];
  double pos = (double)q * (double)(n - 1);
  size_t lo = (size_t)floor(pos), hi = (size_t)ceil(pos);
  double w = pos - (double)lo;
  float dlt = v[hi] - v[lo];
  return (float)((double)v[lo] + (double)dlt * w);
}

static inline int iqrm_target(int lag, int i, int csub) {
  if (lag < 0) return i < csub + lag ? i - lag : csub - 1;
  return i < lag ? 0 : i - lag;
}

/* One IQRM window on the GPU path, run_iqrm_one_window_gpu (iqrm.cu:203-345)
 * with the kernels of iqrm.cu:21-185:
 *  - per channel of [chan_start, chan_end) (the top channel is excluded) the
 *    sum and sum of squares over [t0, t1) in double (exact for integer samples),
 *    mean = sum/W; mode 0 -> x = mean, mode 1 -> x = sqrt(max(0, sumsq/W - mean^2));
 *  - radius = max(1, floor(radius_frac*Csub)), lags of orc_iqrm_lags;
 *  - per lag: lagged difference with edge clipping (make_diff_with_clipping),
 *    sorted; q1/median/q3 by pct(); s = |(q3-q1)/1.349|; lags with s <= 0 are
 *    skipped; flag i when d[i]-med > nsigma*s; recv[i]++, cast[target]++;
 *  - mask[i] = recv[i] > 0 and some flagged lag has cast[target] < recv[i].
 * The parameter clamps of iqrm.hpp:33-37 are applied.  mask_full has nchan
 * entries, zero outside [chan_start, chan_end). */
int orc_iqrm_window_mask(const void* data, int nbits, unsigned nchan, unsigned t0,
                         unsigned t1, unsigned chan_start, unsigned chan_end, int mode,
                         float radius_frac, float nsigma, double geofactor, int variant,
                         uint8_t* mask_full) {
  memset(mask_full, 0, nchan);
  if (radius_frac < 0.0f) radius_frac = 0.0f;
  if (nsigma < 0.0f) nsigma = 0.0f;
  if (!(geofactor > 1.0)) geofactor = 1.5;
  if (chan_start >= chan_end || chan_end > nchan) return 0;
  const unsigned csub = chan_end - chan_start;
  const unsigned W = t1 - t0;
  if (csub == 0 || W == 0) return 0;
  float* x = (float*)malloc(sizeof(float) * csub);
  float* d = (float*)malloc(sizeof(float) * csub);
  float* srt = (float*)malloc(sizeof(float) * csub);
  int* recv = (int*)calloc(csub, sizeof(int));
  int* cast = (int*)calloc(csub, sizeof(int));
  int lags[256];
  uint8_t* flags = NULL;
  int rc = 0;
  if (!x || !d || !srt || !recv || !cast) { rc = 9; goto done; }
  for (unsigned i = 0; i < csub; ++i) {
    uint64_t s = 0, s2 = 0;
    for (unsigned t = t0; t < t1; ++t) {
      uint64_t v = ld(data, nbits, (size_t)t * nchan + chan_start + i);
      s += v;
      s2 += v * v;
    }
    double mean = (double)s / (double)W;
    if (mode == 0) {
      x[i] = (float)mean;
    } else {
      double e2 = (double)s2 / (double)W;
      double var = (variant & ORC_FMA_VAR) ? fma(-mean, mean, e2) : e2 - mean * mean;
      if (var < 0.0) var = 0.0;
      x[i] = (float)sqrt(var);
    }
  }
  {
    int radius = (int)floorf(radius_frac * (float)csub);
    if (radius < 1) radius = 1;
    int nl = orc_iqrm_lags(radius, geofactor, lags, 256);
    if (nl > 256) { rc = 8; goto done; }
    flags = (uint8_t*)calloc((size_t)nl * csub, 1);
    if (!flags) { rc = 9; goto done; }
    for (int l = 0; l < nl; ++l) {
      int lag = lags[l];
      if (lag < 0) {
        int cut = (int)csub + lag;
        float edge = x[cut] - x[csub - 1];
        for (int k = 0; k < (int)csub; ++k) d[k] = k < cut ? x[k] - x[k - lag] : edge;
      } else {
        float edge = x[lag] - x[0];
        for (int k = 0; k < (int)csub; ++k) d[k] = k < lag ? edge : x[k] - x[k - lag];
      }
      memcpy(srt, d, sizeof(float) * csub);
      qsort(srt, csub, sizeof(float), cmp_float);
      float q1 = pct(srt, csub, 0.25f), med = pct(srt, csub, 0.50f), q3 = pct(srt, csub, 0.75f);
      float s;
      if (variant & ORC_RECIP_1349) {
        const float inv = 1.0f / 1.349f;
        s = fabsf((q3 - q1) * inv);
      } else {
        s = fabsf((q3 - q1) / 1.349f);
      }
      if (!(s > 0.f) || !isfinite(s)) continue;
      float thr = nsigma * s;
      for (int i = 0; i < (int)csub; ++i) {
        float val = d[i] - med;
        if (val > thr) {
          flags[(size_t)l * csub + i] = 1;
          recv[i] += 1;
          cast[iqrm_target(lag, i, (int)csub)] += 1;
        }
      }
    }
    for (int i = 0; i < (int)csub; ++i) {
      int ri = recv[i];
      uint8_t m = 0;
      if (ri > 0) {
        for (int l = 0; l < nl; ++l) {
          if (!flags[(size_t)l * csub + i]) continue;
          if (cast[iqrm_target(lags[l], i, (int)csub)] < ri) { m = 1; break; }
        }
      }
      mask_full[chan_start + i] = m;
    }
  }
done:
  free(x); free(d); free(srt); free(recv); free(cast); free(flags);
  return rc;
}

/* RfiMarker<T>::mask (rfimarker.cu:309-390): for each window, zero the flagged
 * channels over [min(t0,nsamp), min(t1,nsamp)). */
void orc_apply_window_masks(void* data, int nbits, unsigned nchan, unsigned nsamp, int nwin,
                            const unsigned* t0, const unsigned* t1, const uint8_t* masks) {
  for (int w = 0; w < nwin; ++w) {
    unsigned a = t0[w] < nsamp ? t0[w] : nsamp;
    unsigned b = t1[w] < nsamp ? t1[w] : nsamp;
    if (a >= b) continue;
    for (unsigned ch = 0; ch < nchan; ++ch) {
      if (!masks[(size_t)w * nchan + ch]) continue;
      for (unsigned t = a; t < b; ++t) st(data, nbits, (size_t)t * nchan + ch, 0);
    }
  }
}

/* The zero-DM call as the reference makes it, dedispered.cu:1107
 * (rfi_marker.zero_dm_filter(d, chan_start, chan_end, down_ndata)): with four
 * arguments it resolves to the overload zero_dm_filter(T*, num_channels,
 * num_samples, float alpha, ...) of rfimarker.h:32-37, i.e. num_channels =
 * chan_start, num_samples = chan_end, alpha = (float)down_ndata.  That overload
 * (rfimarker.cu:130-169) returns at once when num_channels == 0; otherwise it
 * reads the first chan_start*chan_end elements as [chan_end][chan_start]
 * and, per row, subtracts alpha * (float mean of the non-zero values),
 * clipping to [0, vmax] and truncating (kernels rfimarker.cu:32-74, 102-127).
 * The float row sum follows the kernel's order: 256 thread-strided partial sums
 * reduced by a power-of-two tree. */
void orc_zero_dm_callsite(void* data, int nbits, size_t chan_start, size_t chan_end,
                          size_t down_ndata, int variant) {
  const unsigned nc = (unsigned)chan_start;
  const unsigned ns = (unsigned)chan_end;
  const float alpha = (float)down_ndata;
  if (nc == 0 || ns == 0) return;
  const float vmax = (float)vmax_of(nbits);
  float part[256];
  unsigned cnt[256];
  for (unsigned t = 0; t < ns; ++t) {
    for (int k = 0; k < 256; ++k) { part[k] = 0.0f; cnt[k] = 0; }
    for (unsigned ch = 0; ch < nc; ++ch) {
      uint64_t v = ld(data, nbits, (size_t)t * nc + ch);
      if (v) { part[ch % 256] += (float)v; cnt[ch % 256] += 1; }
    }
    for (int s = 128; s > 0; s >>= 1)
      for (int k = 0; k < s; ++k) { part[k] += part[k + s]; cnt[k] += cnt[k + s]; }
    float mean = cnt[0] ? part[0] / (float)cnt[0] : 0.0f;
    for (unsigned ch = 0; ch < nc; ++ch) {
      size_t idx = (size_t)t * nc + ch;
      float v = (float)ld(data, nbits, idx);
      float r;
      if (variant & ORC_FMA_ZDM) r = fmaf(-alpha, mean, v);
      else { float delta = alpha * mean; r = v - delta; }
      if (r < 0.0f) r = 0.0f;
      if (r > vmax) r = vmax;
      st(data, nbits, idx, (uint64_t)r);
    }
  }
}

/* Zero-DM over a channel range with an exact integer mean (the intended range
 * semantics of rfimarker.cu:172-305 with alpha = 1 and clipping at zero): per
 * sample t, over the channels of [chan_start, chan_end), s = sum and c = count of
 * the non-zero values; when c > 0 every value there becomes max(0, v - ceil(s/c)),
 * which equals trunc(max(0, v - s/c)) exactly. */
void orc_zero_dm_range_exact(void* data, int nbits, unsigned nchan, unsigned nsamp,
                             unsigned chan_start, unsigned chan_end) {
  if (chan_end > nchan) chan_end = nchan;
  if (chan_start >= chan_end) return;
  for (unsigned t = 0; t < nsamp; ++t) {
    uint64_t s = 0, c = 0;
    for (unsigned ch = chan_start; ch < chan_end; ++ch) {
      uint64_t v = ld(data, nbits, (size_t)t * nchan + ch);
      if (v) { s += v; c += 1; }
    }
    if (!c) continue;
    uint64_t m = (s + c - 1) / c;
    for (unsigned ch = chan_start; ch < chan_end; ++ch) {
      size_t idx = (size_t)t * nchan + ch;
      uint64_t v = ld(data, nbits, idx);
      st(data, nbits, idx, v > m ? v - m : 0);
    }
  }
}

/* RfiMarker<T>::mark_rfi (rfimarker.cu:469-488, kernel :9-30): zero every listed
 * channel that is inside [0, nchan) for all samples. */
void orc_mark_channels(void* data, int nbits, unsigned nchan, unsigned nsamp, const int* bad,
                       int nbad) {
  for (int b = 0; b < nbad; ++b) {
    int ch = bad[b];
    if (ch < 0 || (unsigned)ch >= nchan) continue;
    for (unsigned t = 0; t < nsamp; ++t) st(data, nbits, (size_t)t * nchan + (unsigned)ch, 0);
  }
}
