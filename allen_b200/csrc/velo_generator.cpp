/*
 * Seeded synthetic VELO events in Allen's raw-bank layout (VP super-pixel banks).
 *
 * Stands in for the LHCb minimum-bias / signal Monte Carlo samples the reference
 * validates on, which are not available.  The detector is the one described by a
 * velo_geometry.bin blob (52 modules, 208 sensors of 3 chips x 256 x 256 pixels;
 * format read by device/event_model/velo/include/ClusteringDefinitions.cuh:164-197).
 *
 * Physics model (per event):
 *   - primary vertices ~ Poisson(nu), nu fixed or drawn uniformly in [nu_min, nu_max];
 *     beam spot Gaussian (sigma_xy, sigma_z);
 *   - charged tracks per vertex ~ Poisson(tracks_per_pv), eta ~ U[eta_min, eta_max],
 *     phi ~ U[0, 2pi), straight lines;
 *   - one hit per crossed sensor with probability hit_efficiency, displaced by a
 *     Gaussian of sigma scatter_sigma in x and y;
 *   - charge sharing: a neighbour column/row joins the cluster when the hit lies within
 *     `share_fraction` of the pixel edge (1, 2, 3 or 4 pixel clusters);
 *   - noise pixels ~ Poisson(noise_rate * pixels) per sensor, uniform on the sensor.
 *
 * Encoding (Allen layout, main/src/Transpose.cpp:333-425; SP word bits per
 * device/velo/mask_clustering/src/EstimateInputSize.cu:29-40):
 *   word = isolated << 31 | (v4: sensor-in-pair << 23) | sp_col << 14 | sp_row << 8 | pattern,
 *   pattern bit (col & 1) * 4 + (row & 3); the isolated flag is set iff none of the eight
 *   neighbouring super pixels of the same sensor is present.
 *   v2/v3: one bank per sensor (sourceID = sensor, count word first);
 *   v4   : one bank per sensor pair (sourceID = pair), no count word.
 *
 * Truth: every signal pixel is recorded with its channel id and owning particle, and
 * every particle with its vertex, eta, phi and the number of distinct modules hit.
 * Each event draws from its own random stream (seed, event index), so the output does
 * not depend on the number of threads.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/velo_generator.h"

namespace {
  constexpr unsigned n_modules = 52;
  constexpr unsigned n_sensors = 208;
  constexpr unsigned n_cols = 768;
  constexpr unsigned n_rows = 256;
  constexpr float pixel_size = 0.055f;
  constexpr double two_pi = 6.283185307179586;

  struct Geometry {
    float module_zs[n_modules];
    float local_x[n_cols];
    float x_pitch[n_cols];
    float ltg[n_sensors * 12];
    double col_edge[n_cols + 1];
  };

  bool parse_geometry(const char* blob, size_t size, Geometry& g)
  {
    const char* p = blob;
    const char* end = blob + size;
    auto read_array = [&](size_t n, float* dst) {
      if (p + sizeof(uint64_t) > end) return false;
      uint64_t count;
      std::memcpy(&count, p, sizeof(count));
      p += sizeof(count);
      if (count != n || p + n * sizeof(float) > end) return false;
      std::memcpy(dst, p, n * sizeof(float));
      p += n * sizeof(float);
      return true;
    };
    if (!read_array(n_modules, g.module_zs)) return false;
    if (!read_array(n_cols, g.local_x)) return false;
    if (!read_array(n_cols, g.x_pitch)) return false;
    if (p + 2 * sizeof(uint64_t) > end) return false;
    uint64_t n_ltg, n_trans;
    std::memcpy(&n_ltg, p, 8);
    std::memcpy(&n_trans, p + 8, 8);
    p += 16;
    if (n_ltg != n_sensors || n_trans != 12 || p + n_sensors * 12 * sizeof(float) > end) return false;
    std::memcpy(g.ltg, p, n_sensors * 12 * sizeof(float));
    // Column c spans [local_x[c] - half a standard pitch, + x_pitch[c]).
    const double offset = 0.5 * g.x_pitch[0];
    for (unsigned c = 0; c < n_cols; ++c)
      g.col_edge[c] = double(g.local_x[c]) - offset;
    g.col_edge[n_cols] = g.col_edge[n_cols - 1] + g.x_pitch[n_cols - 1];
    return true;
  }

  // xoshiro256** seeded through splitmix64.
  struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed)
    {
      for (auto& v : s) {
        seed += 0x9E3779B97F4A7C15ull;
        uint64_t z = seed;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        v = z ^ (z >> 31);
      }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next()
    {
      const uint64_t r = rotl(s[1] * 5, 7) * 9;
      const uint64_t t = s[1] << 17;
      s[2] ^= s[0];
      s[3] ^= s[1];
      s[1] ^= s[2];
      s[0] ^= s[3];
      s[2] ^= t;
      s[3] = rotl(s[3], 45);
      return r;
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double gauss()
    {
      double u1 = uniform();
      while (u1 <= 0.0)
        u1 = uniform();
      return std::sqrt(-2.0 * std::log(u1)) * std::cos(two_pi * uniform());
    }
    unsigned poisson(double mean)
    {
      if (mean <= 0) return 0;
      if (mean > 60) {
        const double v = mean + std::sqrt(mean) * gauss() + 0.5;
        return v < 0 ? 0u : unsigned(v);
      }
      const double l = std::exp(-mean);
      unsigned k = 0;
      double p = uniform();
      while (p > l) {
        ++k;
        p *= uniform();
      }
      return k;
    }
  };

  struct Pixel {
    uint32_t sensor, col, row;
    int32_t particle; // -1 for noise
  };

  struct EventOut {
    std::vector<uint32_t> words;     // event blob as u32 words
    std::vector<uint16_t> bank_sizes;
    std::vector<uint8_t> bank_types;
    std::vector<VeloGenTruthPixel> truth_pixels;
    std::vector<VeloGenParticle> particles;
  };

  void generate_event(const VeloGenConfig& cfg, const Geometry& g, uint64_t seed, unsigned event, EventOut& out)
  {
    Rng rng(seed * 0x100000001B3ull + event * 0x9E3779B97F4A7C15ull + 0x1234567ull);
    std::vector<Pixel> pixels;
    pixels.reserve(8192);

    double nu = cfg.mean_pileup;
    if (cfg.pileup_max > cfg.pileup_min) nu = cfg.pileup_min + (cfg.pileup_max - cfg.pileup_min) * rng.uniform();
    const unsigned n_pv = rng.poisson(nu);

    std::vector<unsigned> module_hit;
    for (unsigned pv = 0; pv < n_pv; ++pv) {
      const double vx = cfg.beam_sigma_xy * rng.gauss();
      const double vy = cfg.beam_sigma_xy * rng.gauss();
      const double vz = cfg.beam_sigma_z * rng.gauss();
      const unsigned n_tracks = rng.poisson(cfg.tracks_per_pv);
      for (unsigned t = 0; t < n_tracks; ++t) {
        const double eta = cfg.eta_min + (cfg.eta_max - cfg.eta_min) * rng.uniform();
        const double phi = two_pi * rng.uniform();
        const double theta = 2.0 * std::atan(std::exp(-eta));
        const double tx = std::tan(theta) * std::cos(phi);
        const double ty = std::tan(theta) * std::sin(phi);
        const int32_t particle = int32_t(out.particles.size());
        module_hit.assign(n_modules, 0);
        unsigned n_hits = 0;
        for (unsigned s = 0; s < n_sensors; ++s) {
          const float* m = g.ltg + 12 * s;
          const double z = m[11];
          if (z <= vz) continue;
          const double gx = vx + tx * (z - vz) + cfg.scatter_sigma * rng.gauss();
          const double gy = vy + ty * (z - vz) + cfg.scatter_sigma * rng.gauss();
          const double dx = gx - m[9], dy = gy - m[10];
          const double lx = m[0] * dx + m[3] * dy;
          const double ly = m[1] * dx + m[4] * dy;
          if (lx < g.col_edge[0] || lx >= g.col_edge[n_cols] || ly < 0 || ly >= n_rows * double(pixel_size)) continue;
          if (rng.uniform() >= cfg.hit_efficiency) continue;
          const unsigned col = unsigned(std::upper_bound(g.col_edge, g.col_edge + n_cols + 1, lx) - g.col_edge) - 1;
          const unsigned row = std::min(n_rows - 1, unsigned(ly / pixel_size));
          const double u = (lx - g.col_edge[col]) / g.x_pitch[col];
          const double v = ly / pixel_size - row;
          int dcol = 0, drow = 0;
          if (u < cfg.share_fraction && col > 0) dcol = -1;
          else if (u > 1.0 - cfg.share_fraction && col + 1 < n_cols) dcol = 1;
          if (v < cfg.share_fraction && row > 0) drow = -1;
          else if (v > 1.0 - cfg.share_fraction && row + 1 < n_rows) drow = 1;
          pixels.push_back({s, col, row, particle});
          if (dcol) pixels.push_back({s, col + dcol, row, particle});
          if (drow) pixels.push_back({s, col, row + drow, particle});
          if (dcol && drow && rng.uniform() >= cfg.drop_corner_fraction)
            pixels.push_back({s, col + dcol, row + drow, particle});
          module_hit[s / 4] = 1;
          ++n_hits;
        }
        unsigned n_mod = 0;
        for (unsigned mh : module_hit)
          n_mod += mh;
        VeloGenParticle pinfo;
        pinfo.pv = pv;
        pinfo.eta = float(eta);
        pinfo.phi = float(phi);
        pinfo.n_hits = n_hits;
        pinfo.n_modules = n_mod;
        out.particles.push_back(pinfo);
      }
    }

    // Noise pixels
    const double pix_per_sensor = double(n_cols) * n_rows;
    for (unsigned s = 0; s < n_sensors; ++s) {
      const unsigned n_noise = rng.poisson(cfg.noise_rate * pix_per_sensor);
      for (unsigned k = 0; k < n_noise; ++k) {
        const unsigned col = unsigned(rng.uniform() * n_cols) % n_cols;
        const unsigned row = unsigned(rng.uniform() * n_rows) % n_rows;
        pixels.push_back({s, col, row, -1});
      }
    }

    // Sort: sensor, col, row; first owner wins for truth.
    std::sort(pixels.begin(), pixels.end(), [](const Pixel& a, const Pixel& b) {
      if (a.sensor != b.sensor) return a.sensor < b.sensor;
      if (a.col != b.col) return a.col < b.col;
      if (a.row != b.row) return a.row < b.row;
      return a.particle > b.particle;
    });
    pixels.erase(
      std::unique(
        pixels.begin(),
        pixels.end(),
        [](const Pixel& a, const Pixel& b) { return a.sensor == b.sensor && a.col == b.col && a.row == b.row; }),
      pixels.end());
    for (const auto& px : pixels) {
      if (px.particle < 0) continue;
      const uint32_t chip = px.col >> 8;
      const uint32_t cid = (px.sensor << 18) | (chip << 16) | ((px.col & 0xFF) << 8) | px.row;
      out.truth_pixels.push_back({(0x2u << 28) | (cid & 0x0FFFFFFFu), uint32_t(px.particle)});
    }

    // Super pixels per sensor
    std::vector<std::vector<uint32_t>> sensor_words(n_sensors);
    {
      size_t i = 0;
      std::vector<uint32_t> keys;
      std::vector<uint8_t> patterns;
      while (i < pixels.size()) {
        const unsigned s = pixels[i].sensor;
        keys.clear();
        patterns.clear();
        for (; i < pixels.size() && pixels[i].sensor == s; ++i) {
          const uint32_t key = ((pixels[i].col >> 1) << 6) | (pixels[i].row >> 2);
          const uint8_t bit = uint8_t(1u << ((pixels[i].col & 1) * 4 + (pixels[i].row & 3)));
          if (!keys.empty() && keys.back() == key) patterns.back() |= bit;
          else {
            keys.push_back(key);
            patterns.push_back(bit);
          }
        }
        // keys are sorted (col-major, then row) because pixels are sorted by col, row
        // and both pixel columns of a super pixel sort next to each other after a merge.
        std::vector<std::pair<uint32_t, uint8_t>> sps;
        for (size_t k = 0; k < keys.size(); ++k)
          sps.push_back({keys[k], patterns[k]});
        std::sort(sps.begin(), sps.end());
        std::vector<std::pair<uint32_t, uint8_t>> merged;
        for (auto& e : sps) {
          if (!merged.empty() && merged.back().first == e.first) merged.back().second |= e.second;
          else merged.push_back(e);
        }
        auto present = [&](int c, int r) {
          if (c < 0 || r < 0 || r > 63 || c > 383) return false;
          const uint32_t key = (uint32_t(c) << 6) | uint32_t(r);
          auto it = std::lower_bound(
            merged.begin(), merged.end(), key, [](const std::pair<uint32_t, uint8_t>& a, uint32_t k) {
              return a.first < k;
            });
          return it != merged.end() && it->first == key;
        };
        for (auto& e : merged) {
          const int c = int(e.first >> 6), r = int(e.first & 0x3F);
          bool neighbour = false;
          for (int dc = -1; dc <= 1 && !neighbour; ++dc)
            for (int dr = -1; dr <= 1 && !neighbour; ++dr)
              if ((dc || dr) && present(c + dc, r + dr)) neighbour = true;
          uint32_t word = (uint32_t(c) << 14) | (uint32_t(r) << 8) | e.second;
          if (!neighbour) word |= 0x80000000u;
          sensor_words[s].push_back(word);
        }
      }
    }

    // Retina clusters (raw_format 1): the pixels of each sensor grouped by 8-connectivity,
    // centroid column and row with a 3-bit (version 2) or 2-bit (versions 3, 4) fraction,
    // in the VPRetinaCluster word layout DecodeRetinaClusters.cu:116-140 reads.
    if (cfg.raw_format == 1) {
      const bool v2 = cfg.bank_version == 2;
      const double q = v2 ? 8.0 : 4.0;
      for (auto& w : sensor_words)
        w.clear();
      size_t i = 0;
      std::unordered_map<uint32_t, unsigned> where;
      std::vector<unsigned> stack;
      while (i < pixels.size()) {
        const unsigned s = pixels[i].sensor;
        size_t j = i;
        where.clear();
        for (; j < pixels.size() && pixels[j].sensor == s; ++j)
          where[(pixels[j].col << 8) | pixels[j].row] = unsigned(j);
        std::vector<char> seen(j - i, 0);
        for (size_t k = i; k < j; ++k) {
          if (seen[k - i]) continue;
          double sc = 0, sr = 0;
          unsigned n = 0;
          stack.assign(1, unsigned(k));
          seen[k - i] = 1;
          while (!stack.empty()) {
            const unsigned m = stack.back();
            stack.pop_back();
            sc += pixels[m].col;
            sr += pixels[m].row;
            ++n;
            for (int dc = -1; dc <= 1; ++dc)
              for (int dr = -1; dr <= 1; ++dr) {
                const int c = int(pixels[m].col) + dc, r = int(pixels[m].row) + dr;
                if ((!dc && !dr) || c < 0 || r < 0 || c >= int(n_cols) || r >= int(n_rows)) continue;
                const auto it = where.find((uint32_t(c) << 8) | uint32_t(r));
                if (it != where.end() && !seen[it->second - i]) {
                  seen[it->second - i] = 1;
                  stack.push_back(it->second);
                }
              }
          }
          const double mc = sc / n, mr = sr / n;
          const uint32_t cx = uint32_t(mc), cy = uint32_t(mr);
          const uint32_t fx = std::min(uint32_t((mc - cx) * q), uint32_t(q) - 1);
          const uint32_t fy = std::min(uint32_t((mr - cy) * q), uint32_t(q) - 1);
          const uint32_t word = v2 ? ((cx << 14) | (fx << 11) | (cy << 3) | fy) : ((cx << 12) | (fx << 10) | (cy << 2) | fy);
          sensor_words[s].push_back(word);
        }
        i = j;
      }
    }

    // Allen event blob
    const bool v4 = cfg.bank_version == 4;
    const unsigned n_banks = v4 ? n_sensors / 2 : n_sensors;
    std::vector<std::vector<uint32_t>> banks(n_banks);
    for (unsigned b = 0; b < n_banks; ++b) {
      auto& d = banks[b];
      if (v4) {
        for (unsigned half = 0; half < 2; ++half)
          for (uint32_t w : sensor_words[2 * b + half])
            d.push_back(w | (half ? (cfg.raw_format == 1 ? 0x400000u : 0x800000u) : 0u));
      }
      else {
        d.push_back(uint32_t(sensor_words[b].size()));
        d.insert(d.end(), sensor_words[b].begin(), sensor_words[b].end());
      }
      // Readout order: the detector does not write a bank's SPs in column order (the
      // 2018 minbias sample has about one bank in nine sorted), so sp_order 1 shuffles them.
      if (cfg.sp_order == 1) {
        const size_t first = v4 ? 0 : 1;
        for (size_t k = d.size(); k > first + 1; --k) {
          const size_t j = first + size_t(rng.next() % (k - first));
          std::swap(d[k - 1], d[j]);
        }
      }
    }
    out.words.clear();
    out.words.push_back(n_banks);
    std::vector<uint32_t> offs(n_banks + 1, 0);
    for (unsigned b = 0; b < n_banks; ++b)
      offs[b + 1] = offs[b] + 4 * uint32_t(1 + banks[b].size());
    out.words.insert(out.words.end(), offs.begin(), offs.end());
    for (unsigned b = 0; b < n_banks; ++b) {
      out.words.push_back(b); // sourceID: sensor (v2/v3) or sensor pair (v4)
      out.words.insert(out.words.end(), banks[b].begin(), banks[b].end());
      out.bank_sizes.push_back(uint16_t(4 * banks[b].size()));
      out.bank_types.push_back(cfg.raw_format == 1 ? 73 : 63); // LHCb::RawBank::VPRetinaCluster or VP
    }
  }

  struct Handle {
    std::vector<EventOut> events;
    uint64_t raw_bytes = 0;
    uint64_t n_truth = 0;
    uint64_t n_particles = 0;
    uint64_t n_sizes = 0;
  };
} // namespace

extern "C" {

void velo_gen_default_config(VeloGenConfig* cfg)
{
  cfg->mean_pileup = 7.6;
  cfg->pileup_min = 0.0;
  cfg->pileup_max = 0.0;
  cfg->tracks_per_pv = 25.0;
  cfg->eta_min = 2.0;
  cfg->eta_max = 5.0;
  cfg->beam_sigma_xy = 0.04;
  cfg->beam_sigma_z = 45.0;
  cfg->hit_efficiency = 0.98;
  cfg->scatter_sigma = 0.01;
  cfg->noise_rate = 1e-5;
  cfg->share_fraction = 0.15;
  cfg->drop_corner_fraction = 0.3;
  cfg->bank_version = 2;
  cfg->sp_order = 1;
  cfg->raw_format = 0;
}

void* velo_gen_create(
  const VeloGenConfig* cfg,
  const char* geometry,
  size_t geometry_size,
  uint64_t seed,
  unsigned first_event,
  unsigned n_events,
  unsigned n_threads)
{
  auto geo = std::make_unique<Geometry>();
  if (!cfg || !geometry || !parse_geometry(geometry, geometry_size, *geo)) return nullptr;
  if (cfg->bank_version != 2 && cfg->bank_version != 3 && cfg->bank_version != 4) return nullptr;
  auto* h = new Handle;
  h->events.resize(n_events);
  if (n_threads == 0) n_threads = std::max(1u, std::thread::hardware_concurrency());
  n_threads = std::min(n_threads, std::max(1u, n_events));
  std::vector<std::thread> workers;
  for (unsigned t = 0; t < n_threads; ++t) {
    workers.emplace_back([&, t] {
      for (unsigned e = t; e < n_events; e += n_threads)
        generate_event(*cfg, *geo, seed, first_event + e, h->events[e]);
    });
  }
  for (auto& w : workers)
    w.join();
  for (auto& e : h->events) {
    h->raw_bytes += 4 * e.words.size();
    h->n_truth += e.truth_pixels.size();
    h->n_particles += e.particles.size();
    h->n_sizes += e.bank_sizes.size();
  }
  return h;
}

void velo_gen_sizes(const void* handle, VeloGenSizes* sizes)
{
  const auto* h = static_cast<const Handle*>(handle);
  const uint64_t n = h->events.size();
  sizes->n_events = n;
  sizes->raw_bytes = h->raw_bytes;
  // u32 offsets header + u16 sizes, rounded up to whole u32 words
  sizes->sizes_words = (n + 1) + (h->n_sizes + 1) / 2;
  // u32 offsets header + u8 types, rounded up to whole u32 words
  sizes->types_words = (n + 1) + (h->n_sizes + 3) / 4;
  sizes->n_truth_pixels = h->n_truth;
  sizes->n_particles = h->n_particles;
}

void velo_gen_copy(
  const void* handle,
  char* raw,
  unsigned* raw_offsets,
  unsigned* raw_sizes,
  unsigned* raw_types,
  VeloGenTruthPixel* truth_pixels,
  unsigned* truth_offsets,
  VeloGenParticle* particles,
  unsigned* particle_offsets)
{
  const auto* h = static_cast<const Handle*>(handle);
  const unsigned n = unsigned(h->events.size());
  uint64_t raw_pos = 0;
  unsigned size_pos = 2 * (n + 1);
  unsigned type_pos = 4 * (n + 1);
  uint64_t truth_pos = 0, particle_pos = 0;
  for (unsigned e = 0; e < n; ++e) {
    const auto& ev = h->events[e];
    if (raw_offsets) raw_offsets[e] = unsigned(raw_pos);
    if (raw) std::memcpy(raw + raw_pos, ev.words.data(), 4 * ev.words.size());
    raw_pos += 4 * ev.words.size();
    if (raw_sizes) {
      raw_sizes[e] = size_pos;
      std::memcpy(reinterpret_cast<uint16_t*>(raw_sizes) + size_pos, ev.bank_sizes.data(), 2 * ev.bank_sizes.size());
    }
    size_pos += unsigned(ev.bank_sizes.size());
    if (raw_types) {
      raw_types[e] = type_pos;
      std::memcpy(reinterpret_cast<uint8_t*>(raw_types) + type_pos, ev.bank_types.data(), ev.bank_types.size());
    }
    type_pos += unsigned(ev.bank_types.size());
    if (truth_offsets) truth_offsets[e] = unsigned(truth_pos);
    if (truth_pixels)
      std::memcpy(truth_pixels + truth_pos, ev.truth_pixels.data(), sizeof(VeloGenTruthPixel) * ev.truth_pixels.size());
    truth_pos += ev.truth_pixels.size();
    if (particle_offsets) particle_offsets[e] = unsigned(particle_pos);
    if (particles)
      std::memcpy(particles + particle_pos, ev.particles.data(), sizeof(VeloGenParticle) * ev.particles.size());
    particle_pos += ev.particles.size();
  }
  if (raw_offsets) raw_offsets[n] = unsigned(raw_pos);
  if (raw_sizes) raw_sizes[n] = size_pos;
  if (raw_types) raw_types[n] = type_pos;
  if (truth_offsets) truth_offsets[n] = unsigned(truth_pos);
  if (particle_offsets) particle_offsets[n] = unsigned(particle_pos);
}

void velo_gen_destroy(void* handle) { delete static_cast<Handle*>(handle); }
}
