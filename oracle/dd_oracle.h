/* ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of astroflow's dedispersion hot path, used only as the
 * parity reference by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
 * The product (astroflow_b200) never links, loads or calls anything here.
 *
 * Parity pin: every function is checked against the reference's own code
 * compiled from source (oracle/_ref: the CPU brute force of include/cpucal.hpp
 * here, and the GPU path of src/core/dedispered.cu, src/core/iqrm.cu,
 * src/rfi/rfimarker.cu on a B200) by tests/test_oracle_pin.py and
 * tests/test_ref_tap_gpu.py, and by the fixtures in tests/golden/.
 *
 * Element types: nbits 8/16/32 selects uint8/uint16/uint32 input samples,
 * laid out time-major, data[t * nchans + ch] (include/data.h, Header).
 */
#ifndef DD_ORACLE_H
#define DD_ORACLE_H
#include <stddef.h>
#include <stdint.h>

/* Variant bits for arithmetic the reference leaves to its compiler flags. */
#define ORC_FMA_DM       1   /* dm = fma(i, step, lo) instead of lo + i*step          */
#define ORC_RECIP_TSAMP  2   /* delay * (1/tsamp) instead of delay / tsamp (CPU path) */
#define ORC_RECIP_1349   4   /* (q3-q1) * (1/1.349f) instead of /1.349f (IQRM)        */
#define ORC_FMA_VAR      8   /* var = fma(-mean, mean, sumsq/W) (IQRM std)            */
#define ORC_FMA_ZDM     16   /* r = fma(-alpha, mean, v) (zero-DM subtract)           */
#define ORC_CPU_EXPAND  32   /* delay = (K*dm)*a - (K*dm)*b (CPU brute force)          */
#define ORC_CPU_EXPFMA  64   /* delay = fma(K*dm, a, -(K*dm)*b) (CPU brute force)      */

void orc_freq_table_header(float fch1, float foff, int nchans, double* freq);
void orc_freq_table_fil(double fch1, double foff, int nchans, double* freq);
int orc_chan_range(const double* freq, int nchans, float freq_start, float freq_end,
                   long* chan_start, long* chan_end);
long orc_dm_steps(float dm_low, float dm_high, float dm_step);

void orc_subband_tables_ieee(const double* freq, long chan_start, long chan_end, float dm_low,
                             float dm_step, long dm_steps, int sb_width, int ndm0, double tsamp,
                             int ds, int variant, int* delay1, int* residual2);
void orc_delay_table_fp64(const double* freq, long chan_start, long chan_end, float dm_low,
                          float dm_step, long ndm, double tsamp, int ds, int* delay);
void orc_cpu_delay_table(const double* freq, long chan_start, long chan_end, float dm_low,
                         float dm_step, long dm_steps, double tsamp, int variant, int* delay);

int orc_bruteforce_cpu(const void* data, int nbits, long ndata, int nchans, const double* freq,
                       double tsamp, float dm_low, float dm_high, float freq_start,
                       float freq_end, float dm_step, int ds, float t_sample, int variant,
                       const int* delay_in, uint64_t* out, long out_cap, long* nslices,
                       long* slice_cols, long slice_cap, long* ndm);

int orc_subband_sums(const void* data, int nbits, long nsamp, int nchans, long chan_start,
                     long chan_end, int sb_width, int ndm0, long dm_steps, const int* delay1,
                     const int* residual2, uint64_t* out);

int orc_time_binning(const void* in, int nbits, long ndata, int nchans, int ds, void* out);

int orc_iqrm_windows(double win_sec, double hop_sec, int include_tail, double tsamp,
                     unsigned nsample, unsigned* t0, unsigned* t1, int cap);
int orc_iqrm_window_mask(const void* data, int nbits, unsigned nchan, unsigned t0,
                         unsigned t1, unsigned chan_start, unsigned chan_end, int mode,
                         float radius_frac, float nsigma, double geofactor, int variant,
                         uint8_t* mask_full);
int orc_iqrm_lags(int radius, double geofactor, int* lags, int cap);

void orc_apply_window_masks(void* data, int nbits, unsigned nchan, unsigned nsamp, int nwin,
                            const unsigned* t0, const unsigned* t1, const uint8_t* masks);
void orc_zero_dm_callsite(void* data, int nbits, size_t chan_start, size_t chan_end,
                          size_t down_ndata, int variant);
void orc_zero_dm_range_exact(void* data, int nbits, unsigned nchan, unsigned nsamp,
                             unsigned chan_start, unsigned chan_end);
void orc_mark_channels(void* data, int nbits, unsigned nchan, unsigned nsamp, const int* bad,
                       int nbad);

#endif
