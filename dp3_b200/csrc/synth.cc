// Seeded synthetic interferometer observations; see synth.h.
#include "synth.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr double kSpeedOfLight = 299792458.0;
constexpr double kPi = 3.14159265358979323846;

// Uniform double in [0, 1) from the top 53 bits.
double Uniform(std::mt19937_64& rng) {
  return double(rng() >> 11) * (1.0 / 9007199254740992.0);
}
// Standard normal via Box-Muller on two uniforms in (0, 1].
double Normal(std::mt19937_64& rng) {
  const double u1 = 1.0 - Uniform(rng);
  const double u2 = Uniform(rng);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
}

uint64_t SplitMix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Complex normal (sigma per component) from a counter.
std::complex<double> HashComplexNormal(uint64_t seed, uint64_t counter) {
  const uint64_t a = SplitMix64(seed ^ SplitMix64(2 * counter));
  const uint64_t b = SplitMix64(seed ^ SplitMix64(2 * counter + 1));
  const double u1 = 1.0 - double(a >> 11) * (1.0 / 9007199254740992.0);
  const double u2 = double(b >> 11) * (1.0 / 9007199254740992.0);
  const double r = std::sqrt(-2.0 * std::log(u1));
  return {r * std::cos(2.0 * kPi * u2), r * std::sin(2.0 * kPi * u2)};
}

struct Sky {
  std::vector<double> enu;                  // [n_st][3]
  std::vector<double> l, m, nm1, flux;      // [n_dir * n_src]
};

Sky MakeSky(const synth_config& c) {
  Sky s;
  std::mt19937_64 rng(c.sky_seed);
  s.enu.resize(size_t(c.n_stations) * 3);
  if (c.layout == 0) {
    for (uint32_t i = 0; i < c.n_stations; ++i) {
      const double r = c.radius_m * std::sqrt(Uniform(rng));
      const double th = 2.0 * kPi * Uniform(rng);
      s.enu[3 * i] = r * std::cos(th);
      s.enu[3 * i + 1] = r * std::sin(th);
      s.enu[3 * i + 2] = 0.0;
    }
  } else {
    // Three logarithmic spiral arms from r_min to radius_m, 1.5 turns each,
    // with 2 % radial jitter.
    const double r_min = std::max(25.0, c.radius_m * 1e-3);
    for (uint32_t i = 0; i < c.n_stations; ++i) {
      const uint32_t arm = i % 3;
      const uint32_t k = i / 3;
      const uint32_t per_arm = (c.n_stations + 2 - arm) / 3;
      const double frac = per_arm > 1 ? double(k) / double(per_arm - 1) : 0.0;
      const double r = r_min * std::pow(c.radius_m / r_min, frac) *
                       (1.0 + 0.02 * (Uniform(rng) - 0.5));
      const double th = arm * 2.0 * kPi / 3.0 + 1.5 * 2.0 * kPi * frac;
      s.enu[3 * i] = r * std::cos(th);
      s.enu[3 * i + 1] = r * std::sin(th);
      s.enu[3 * i + 2] = 0.0;
    }
  }
  const size_t n = size_t(c.n_directions) * c.n_sources;
  s.l.resize(n);
  s.m.resize(n);
  s.nm1.resize(n);
  s.flux.resize(n);
  const double rmax = c.max_offset_deg * kPi / 180.0;
  const double lmin = std::log(c.flux_min_jy), lmax = std::log(c.flux_max_jy);
  for (size_t i = 0; i < n; ++i) {
    const double r = rmax * std::sqrt(Uniform(rng));
    const double ps = 2.0 * kPi * Uniform(rng);
    s.l[i] = r * std::cos(ps);
    s.m[i] = r * std::sin(ps);
    s.nm1[i] = std::sqrt(1.0 - s.l[i] * s.l[i] - s.m[i] * s.m[i]) - 1.0;
    s.flux[i] = std::exp(lmin + (lmax - lmin) * Uniform(rng));
  }
  return s;
}

std::vector<double> Frequencies(const synth_config& c) {
  std::vector<double> f(c.n_channels);
  const double w = (c.freq_hi_hz - c.freq_lo_hz) / c.n_channels;
  for (uint32_t i = 0; i < c.n_channels; ++i) f[i] = c.freq_lo_hz + w * (i + 0.5);
  return f;
}

// Station UVW (metres) at hour angle H for declination dec, from local ENU at
// latitude lat (equatorial frame: X towards H = 0 on the equator, Z to the
// north celestial pole).
void StationUvw(const std::vector<double>& enu, size_t n_st, double H,
                double dec, double lat, std::vector<double>& uvw) {
  uvw.resize(n_st * 3);
  const double sl = std::sin(lat), cl = std::cos(lat);
  const double sH = std::sin(H), cH = std::cos(H);
  const double sd = std::sin(dec), cd = std::cos(dec);
  for (size_t i = 0; i < n_st; ++i) {
    const double e = enu[3 * i], n = enu[3 * i + 1], u = enu[3 * i + 2];
    const double X = -sl * n + cl * u;
    const double Y = e;
    const double Z = cl * n + sl * u;
    uvw[3 * i] = sH * X + cH * Y;
    uvw[3 * i + 1] = -sd * cH * X + sd * sH * Y + cd * Z;
    uvw[3 * i + 2] = cd * cH * X - cd * sH * Y + sd * Z;
  }
}

}  // namespace

extern "C" {

int synth_layout(const synth_config* cfg, double* enu) {
  if (!cfg || !enu) return 1;
  const Sky s = MakeSky(*cfg);
  std::memcpy(enu, s.enu.data(), s.enu.size() * sizeof(double));
  return 0;
}

int synth_station_uvw(const synth_config* cfg, double* uvw) {
  if (!cfg || !uvw) return 1;
  const synth_config& c = *cfg;
  const Sky s = MakeSky(c);
  const double dec = c.dec_deg * kPi / 180.0, lat = c.lat_deg * kPi / 180.0;
  const double omega = 7.2921150e-5;  // as synth_observe
  std::vector<double> one;
  for (uint32_t t = 0; t < c.n_times; ++t) {
    StationUvw(s.enu, c.n_stations, omega * (c.start_time_s + t * c.time_step_s), dec, lat,
               one);
    std::memcpy(uvw + size_t(t) * c.n_stations * 3, one.data(), one.size() * sizeof(double));
  }
  return 0;
}

int synth_sky(const synth_config* cfg, double* lmn, double* flux) {
  if (!cfg || !lmn || !flux) return 1;
  const Sky s = MakeSky(*cfg);
  for (size_t k = 0; k < s.l.size(); ++k) {
    lmn[3 * k] = s.l[k];
    lmn[3 * k + 1] = s.m[k];
    lmn[3 * k + 2] = s.nm1[k] + 1.0;
    flux[k] = s.flux[k];
  }
  return 0;
}

int synth_frequencies(const synth_config* cfg, double* freqs) {
  if (!cfg || !freqs) return 1;
  const std::vector<double> f = Frequencies(*cfg);
  std::memcpy(freqs, f.data(), f.size() * sizeof(double));
  return 0;
}

uint64_t synth_n_baselines(const synth_config* cfg) {
  return cfg ? uint64_t(cfg->n_stations) * (cfg->n_stations - 1) / 2 : 0;
}

int synth_gains(const synth_config* cfg, uint64_t seed, double amp_sigma,
                double delay_sigma_ns, double* gains) {
  if (!cfg || !gains) return 1;
  const synth_config& c = *cfg;
  std::mt19937_64 rng(seed);
  const std::vector<double> f = Frequencies(c);
  const double f_mid = 0.5 * (c.freq_lo_hz + c.freq_hi_hz);
  const size_t n = size_t(c.n_stations) * c.n_directions * 2;
  std::vector<double> amp(n), ph(n), tau(n);
  for (size_t i = 0; i < n; ++i) {
    amp[i] = std::exp(amp_sigma * Normal(rng));
    ph[i] = kPi * (2.0 * Uniform(rng) - 1.0);
    tau[i] = delay_sigma_ns * 1e-9 * Normal(rng);
  }
  for (uint32_t ch = 0; ch < c.n_channels; ++ch)
    for (size_t i = 0; i < n; ++i) {
      const double p = ph[i] + 2.0 * kPi * tau[i] * (f[ch] - f_mid);
      gains[2 * (ch * n + i)] = amp[i] * std::cos(p);
      gains[2 * (ch * n + i) + 1] = amp[i] * std::sin(p);
    }
  return 0;
}

int synth_observe(const synth_config* cfg, uint32_t n_cb,
                  const uint32_t* cb_channels, const double* gains,
                  float** data, float** model, uint32_t* antenna1,
                  uint32_t* antenna2) {
  if (!cfg || !cb_channels || !antenna1 || !antenna2) return 1;
  const synth_config& c = *cfg;
  if (data && !gains) return 1;
  std::vector<uint32_t> cb_begin(n_cb + 1, 0);
  for (uint32_t i = 0; i < n_cb; ++i) cb_begin[i + 1] = cb_begin[i] + cb_channels[i];
  if (cb_begin[n_cb] != c.n_channels) return 2;
  const Sky sky = MakeSky(c);
  const std::vector<double> freqs = Frequencies(c);
  const size_t n_st = c.n_stations, n_dir = c.n_directions, n_src = c.n_sources;
  const size_t n_ch = c.n_channels;
  const size_t n_bl = n_st * (n_st - 1) / 2;
  std::vector<uint32_t> bl_p(n_bl), bl_q(n_bl);
  {
    size_t b = 0;
    for (uint32_t p = 0; p < n_st; ++p)
      for (uint32_t q = p + 1; q < n_st; ++q, ++b) {
        bl_p[b] = p;
        bl_q[b] = q;
        antenna1[b] = p;
        antenna2[b] = q;
      }
  }
  const double dec = c.dec_deg * kPi / 180.0, lat = c.lat_deg * kPi / 180.0;
  const double omega = 7.2921150e-5;  // earth rotation, rad / s
  const double df = n_ch > 1 ? freqs[1] - freqs[0] : 0.0;
  const double two_pi_c = 2.0 * kPi / kSpeedOfLight;

  for (uint32_t t = 0; t < c.n_times; ++t) {
    const double H = omega * (c.start_time_s + t * c.time_step_s);
    std::vector<double> uvw;
    StationUvw(sky.enu, n_st, H, dec, lat, uvw);
    // station phase slopes per source: phi_p (radians per Hz)
    std::vector<double> phi(n_st * n_dir * n_src);
    for (size_t p = 0; p < n_st; ++p)
      for (size_t k = 0; k < n_dir * n_src; ++k)
        phi[p * n_dir * n_src + k] =
            two_pi_c * (uvw[3 * p] * sky.l[k] + uvw[3 * p + 1] * sky.m[k] +
                        uvw[3 * p + 2] * sky.nm1[k]);
#pragma omp parallel
    {
      std::vector<std::complex<double>> vis(n_dir * n_ch);
#pragma omp for schedule(dynamic, 64)
      for (size_t b = 0; b < n_bl; ++b) {
        const size_t p = bl_p[b], q = bl_q[b];
        std::fill(vis.begin(), vis.end(), std::complex<double>(0.0, 0.0));
        for (size_t d = 0; d < n_dir; ++d) {
          std::complex<double>* v = &vis[d * n_ch];
          for (size_t s = 0; s < n_src; ++s) {
            const size_t k = d * n_src + s;
            const double dphi = phi[q * n_dir * n_src + k] - phi[p * n_dir * n_src + k];
            const double I = sky.flux[k];
            // exp(i dphi nu) by rotation across channels, restarted per block
            for (uint32_t cb = 0; cb < n_cb; ++cb) {
              const uint32_t c0 = cb_begin[cb], c1 = cb_begin[cb + 1];
              if (c0 == c1) continue;
              std::complex<double> z = std::polar(I, dphi * freqs[c0]);
              const std::complex<double> step = std::polar(1.0, dphi * df);
              for (uint32_t ch = c0; ch < c1; ++ch) {
                v[ch] += z;
                z *= step;
              }
            }
          }
        }
        for (uint32_t cb = 0; cb < n_cb; ++cb) {
          const uint32_t c0 = cb_begin[cb], c1 = cb_begin[cb + 1];
          const size_t w = c1 - c0;
          const size_t nv = size_t(c.n_times) * n_bl * w;
          const size_t vbase = (size_t(t) * n_bl + b) * w;
          for (uint32_t ch = c0; ch < c1; ++ch) {
            const size_t vi = vbase + (ch - c0);
            if (model && model[cb]) {
              for (size_t d = 0; d < n_dir; ++d) {
                float* o = model[cb] + ((d * nv) + vi) * 4;
                const std::complex<double> m = vis[d * n_ch + ch];
                o[0] = float(m.real());
                o[1] = float(m.imag());
                o[2] = float(m.real());
                o[3] = float(m.imag());
              }
            }
            if (data && data[cb]) {
              float* o = data[cb] + vi * 4;
              for (int pol = 0; pol < 2; ++pol) {
                std::complex<double> acc(0.0, 0.0);
                for (size_t d = 0; d < n_dir; ++d) {
                  const double* gp = gains + 2 * (((ch * n_st + p) * n_dir + d) * 2 + pol);
                  const double* gq = gains + 2 * (((ch * n_st + q) * n_dir + d) * 2 + pol);
                  acc += std::complex<double>(gp[0], gp[1]) * vis[d * n_ch + ch] *
                         std::conj(std::complex<double>(gq[0], gq[1]));
                }
                const uint64_t counter =
                    ((uint64_t(t) * n_bl + b) * n_ch + ch) * 2 + pol;
                acc += c.noise_sigma_jy * HashComplexNormal(c.noise_seed, counter);
                o[2 * pol] = float(acc.real());
                o[2 * pol + 1] = float(acc.imag());
              }
            }
          }
        }
      }
    }
  }
  return 0;
}

}  // extern "C"
