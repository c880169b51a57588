/*
 * Seeded synthetic interferometer observations for the solver benchmarks.
 *
 * Station layouts, earth-rotation UVW, point-source sky models and smooth
 * complex gains; model visibilities follow the point-source phase equation
 * used by DP3's predict (base/Simulator.cc:477-520, visibility product
 * :200-245): V_pq = sum_src I exp(i (phi_q - phi_p) nu), with
 * phi_p = 2 pi / c (u_p l + v_p m + w_p (n - 1)). Visibilities are built in
 * FP64 and stored as complex64 XX/YY (unpolarized sources: XX = YY = I), in
 * the layout of DP3's regular SolveData constructor
 * (ddecal/gain_solvers/SolveData.cc:77-188): per channel block, visibility
 * index (t * n_baselines + b) * n_block_channels + c.
 *
 * Randomness: sky, stations and gains come from std::mt19937_64 streams with
 * explicit transforms (no implementation-defined distributions); noise is a
 * counter-based hash of (seed, time, baseline, channel, polarization), so the
 * output does not depend on the number of threads.
 */
#ifndef DP3B200_SYNTH_H
#define DP3B200_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint32_t n_stations;
  uint32_t layout;        /* 0 = uniform disk, 1 = 3-arm log spiral */
  double radius_m;
  uint32_t n_directions;
  uint32_t n_sources;     /* per direction */
  double max_offset_deg;  /* sources within this radius of the phase centre */
  double flux_min_jy;     /* log-uniform flux range */
  double flux_max_jy;
  uint32_t n_channels;
  double freq_lo_hz;      /* band edges; channel centres are evenly spaced */
  double freq_hi_hz;
  uint32_t n_times;
  double time_step_s;
  double start_time_s;    /* of the first time step, hour angle 0 at t = 0 */
  double dec_deg;
  double lat_deg;
  double noise_sigma_jy;  /* per real / imaginary component */
  uint64_t sky_seed;      /* stations and sources */
  uint64_t noise_seed;
} synth_config;

/* Station positions in local east/north/up metres, [n_stations][3]. */
int synth_layout(const synth_config* cfg, double* enu);

/* True gains [n_channels][n_stations][n_directions][2 pol] complex128:
 * exp(N(0, amp_sigma)) * exp(i U(-pi, pi)) * exp(2 pi i tau (nu - nu_mid)),
 * tau ~ N(0, delay_sigma_ns) per station, direction and polarization. */
int synth_gains(const synth_config* cfg, uint64_t seed, double amp_sigma,
                double delay_sigma_ns, double* gains);

/* Station UVW (m) of each time step, [n_times][n_stations][3] (the UVW
 * synth_observe uses). */
int synth_station_uvw(const synth_config* cfg, double* uvw);

/* The point-source sky: lmn [n_directions * n_sources][3] (l, m, n) and the
 * Stokes I flux [n_directions * n_sources] (Jy), direction-major. */
int synth_sky(const synth_config* cfg, double* lmn, double* flux);

/* Channel centre frequencies [n_channels]. */
int synth_frequencies(const synth_config* cfg, double* freqs);

/* Number of cross-correlation baselines: n (n - 1) / 2, ordered
 * (0,1), (0,2), ..., (1,2), ... */
uint64_t synth_n_baselines(const synth_config* cfg);

/* Fills the antenna arrays [n_baselines] and, per channel block cb (with
 * cb_channels[cb] channels, consecutive), data[cb] float32
 * [n_times*n_baselines*cb_channels][2][2] and model[cb] float32
 * [n_directions][same][2][2]. data = sum_d g_p M_d conj(g_q) + noise, with
 * gains [n_channels][n_stations][n_directions][2] (complex128). Any of
 * data / model may be NULL to skip it. */
int synth_observe(const synth_config* cfg, uint32_t n_channel_blocks,
                  const uint32_t* cb_channels, const double* gains,
                  float** data, float** model, uint32_t* antenna1,
                  uint32_t* antenna2);

#ifdef __cplusplus
}
#endif

#endif
