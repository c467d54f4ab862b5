// Brute-force delay table in the arithmetic of the reference's CPU path.
//
// cpucal::dedispered_fil_omp (include/cpucal.hpp:119-132) computes, per DM trial
// `step` and channel ch of [chan_start, chan_end),
//
//   dm    = dm_low + step*dm_step                                  (float)
//   delay = 4148.808f*dm*(1/(f*f) - 1/(ref*ref)),  f = float(freq[ch]) (float)
//   table = (int) round(delay / tsamp)                              (double)
//
// and the reference builds that loop with -Ofast -ffast-math -mfma and AVX2
// (CMakeLists.txt:116-118).  Under those flags the compiler contracts the DM
// into a fused multiply-add, vectorises the reciprocals 1/(f*f) as an
// approximate reciprocal refined by one Newton step, and evaluates the rest
// in vector registers; a few entries per ten thousand then land on the other
// side of a rounding tie from the same expression evaluated in IEEE arithmetic.
// This translation unit is compiled with the reference's host flags, and the
// loop below has the same shape, types and operand order (a per-DM outer loop,
// an inner loop over the band's channels with unit stride, int stores), so
// the compiler makes the same choices and the table equals the reference
// build's entry for entry on the same host CPU.  Nothing here restates the
// compiler's reciprocal sequence.
#include <cmath>
#include <cstddef>
#include <cstdint>

namespace dd {

void brute_delay_table_fastmath(const double* freq, size_t chan_start, size_t chan_end,
                                float dm_low, float dm_step, size_t dm_steps,
                                float ref_freq_value, double tsamp, int32_t* table) {
  const size_t nc = chan_end - chan_start;
  for (size_t step = 0; step < dm_steps; ++step) {
    const float dm = dm_low + step * dm_step;
    int32_t* row = table + step * nc;
    for (size_t ch = chan_start; ch < chan_end; ++ch) {
      const float f = freq[ch];
      const float delay = 4148.808f * dm * (1.0f / (f * f) - 1.0f / (ref_freq_value * ref_freq_value));
      row[ch - chan_start] = static_cast<int>(std::round(delay / tsamp));
    }
  }
}

}  // namespace dd
