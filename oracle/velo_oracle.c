/*
 * ORACLE - test infrastructure, not product code.
 *
 * A plain-C, single-threaded restatement of the reference's VELO super-pixel chain
 * (Allen veloSP: configuration/python/AllenConf/velo_reconstruction.py:72-292),
 * written against the semantics of the reference's CPU build (TARGET_DEVICE_CPU:
 * blockDim = 1, atomics are sequential read-modify-writes,
 * backend/include/CPUBackend.h:97-114).  Only the tests, the smoke check and the
 * benchmark's CPU-baseline leg use it, as the checker; the CUDA library never
 * calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks this file against the reference's
 * own kernels compiled as CPU C++ (oracle/_ref, oracle/ref_driver.cpp) on real and
 * generated events, and against the reference outputs committed in tests/golden/.
 *
 * Floating point follows the reference's expression order with no contraction
 * (built with -ffp-contract=off); the float-to-int16 phi conversion goes through a
 * 32-bit integer exactly like the x86 code the reference compiles to.
 */
#include <math.h>
#include <pthread.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "velo_cpu_api.h"

#define N_MODULES 52u
#define N_MODULE_PAIRS 26u
#define N_SENSORS 208u
#define N_COLS 768u
#define MAX_TRACK_SIZE 26u
#define MAX_TTF 2048u
#define MIN_CONTAINER 10u
#define ELEMENT_SIZE 18u /* u32 id + 3 x f32 + i16 phi (CPU build: half_t == float) */

static const float tracks_per_cluster = 0.34f; /* VeloDefinitions.cuh:23 */
static const float pixel_size = 0.055f;        /* VeloDefinitions.cuh:30 */
static const float pi_f = 3.141592654f;        /* BackendCommonInterface.h:49 */
static const float param_w = 6400.f;           /* VeloDefinitions.cuh:35 */

typedef struct {
  float module_zs[N_MODULES];
  float local_x[N_COLS];
  float x_pitch[N_COLS];
  float ltg[N_SENSORS * 12];
} Geometry;

/* --------------------------------------------------------------------------------
 * Named output buffers (Allen argument names).
 * ------------------------------------------------------------------------------ */
#define MAX_BUFFERS 48
typedef struct {
  char name[64];
  void* p;
  size_t n;
} Buffer;
typedef struct {
  Buffer b[MAX_BUFFERS];
  int count;
} Result;

static void* make(Result* r, const char* name, size_t nbytes)
{
  size_t alloc = nbytes < 64 ? 64 : ((nbytes + 63) / 64) * 64;
  void* p = aligned_alloc(64, alloc);
  memset(p, 0, alloc);
  Buffer* b = &r->b[r->count++];
  strncpy(b->name, name, sizeof(b->name) - 1);
  b->name[sizeof(b->name) - 1] = 0;
  b->p = p;
  b->n = nbytes;
  return p;
}

/* --------------------------------------------------------------------------------
 * Inputs: geometry blob (ClusteringDefinitions.cuh:164-197) and raw banks
 * (ClusteringDefinitions.cuh:61-144, MEPTools.h:26-53).
 * ------------------------------------------------------------------------------ */
static int parse_geometry(const char* blob, size_t size, Geometry* g)
{
  const char* p = blob;
  const char* end = blob + size;
  uint64_t n;
#define READ_ARRAY(N, DST)                                      \
  if (p + 8 > end) return 0;                                    \
  memcpy(&n, p, 8);                                             \
  p += 8;                                                       \
  if (n != (N) || p + (N) * sizeof(float) > end) return 0;      \
  memcpy((DST), p, (N) * sizeof(float));                        \
  p += (N) * sizeof(float);
  READ_ARRAY(N_MODULES, g->module_zs)
  READ_ARRAY(N_COLS, g->local_x)
  READ_ARRAY(N_COLS, g->x_pitch)
#undef READ_ARRAY
  uint64_t n_ltg, n_trans;
  if (p + 16 > end) return 0;
  memcpy(&n_ltg, p, 8);
  memcpy(&n_trans, p + 8, 8);
  p += 16;
  if (n_ltg != N_SENSORS || n_trans != 12 || p + N_SENSORS * 12 * sizeof(float) > end) return 0;
  memcpy(g->ltg, p, N_SENSORS * 12 * sizeof(float));
  return 1;
}

typedef struct {
  uint32_t n_banks;
  const uint32_t* bank_offsets;
  const char* payload;
  const uint16_t* sizes;
  const uint8_t* types;
} RawEvent;

typedef struct {
  uint32_t source_id;
  uint32_t count;
  const uint32_t* word;
  uint16_t size;
  uint16_t type;
} RawBank;

static RawEvent raw_event(const VeloCpuInput* in, unsigned event)
{
  RawEvent r;
  const char* ev = in->raw + in->raw_offsets[event];
  memcpy(&r.n_banks, ev, 4);
  r.bank_offsets = (const uint32_t*) (ev + 4);
  r.payload = ev + 4 + 4 * (r.n_banks + 1);
  r.sizes = (const uint16_t*) in->raw_sizes + in->raw_sizes[event];
  r.types = (const uint8_t*) in->raw_types + in->raw_types[event];
  return r;
}

static RawBank raw_bank(const RawEvent* e, unsigned i, int version)
{
  RawBank b;
  const char* p = e->payload + e->bank_offsets[i];
  memcpy(&b.source_id, p, 4);
  p += 4;
  b.count = 0;
  if (version == 2 || version == 3) {
    memcpy(&b.count, p, 4);
    p += 4;
  }
  b.word = (const uint32_t*) p;
  b.size = e->sizes[i];
  b.type = e->types[i];
  return b;
}

static bool is_velo_bank(const RawBank* b) { return b->type == 63 || b->type == 8; }
static uint32_t sensor_pair(const RawBank* b) { return b->source_id & 0x1FFu; }
static uint32_t sensor_index0(const RawBank* b) { return (b->source_id & 0x1FFu) << 1; }
static uint32_t sensor_index1(const RawBank* b) { return ((b->source_id & 0x1FFu) << 1) | 1u; }
static uint32_t bank_n_sp(const RawBank* b, int version) { return (version == 2 || version == 3) ? b->count : b->size / 4u; }

/* ClusteringDefinitions.cuh:200-216, LHCbID.cuh:36-39 */
static uint32_t channel_id(uint32_t sensor, uint32_t chip, uint32_t col, uint32_t row)
{
  return (sensor << 18) | (chip << 16) | (col << 8) | row;
}
static uint32_t lhcb_id(uint32_t cid) { return ((2u << 28) & 0xF0000000u) | (cid & 0x0FFFFFFFu); }

/* --------------------------------------------------------------------------------
 * Cluster container view (VeloEventModel.cuh:92-189, half_t == float):
 * id[N] u32 | xyz[3N] f32 interleaved | phi[N] i16, N = total size, element at offset+i.
 * ------------------------------------------------------------------------------ */
typedef struct {
  char* base;
  unsigned total;
  unsigned offset;
} Clusters;

static uint32_t c_id(const Clusters* c, unsigned i) { return ((const uint32_t*) c->base)[c->offset + i]; }
static float c_x(const Clusters* c, unsigned i) { return ((const float*) c->base)[c->total + 3 * (c->offset + i)]; }
static float c_y(const Clusters* c, unsigned i) { return ((const float*) c->base)[c->total + 3 * (c->offset + i) + 1]; }
static float c_z(const Clusters* c, unsigned i) { return ((const float*) c->base)[c->total + 3 * (c->offset + i) + 2]; }
static int16_t c_phi(const Clusters* c, unsigned i) { return ((const int16_t*) c->base)[8u * c->total + c->offset + i]; }
static const int16_t* c_phi_begin(const Clusters* c) { return ((const int16_t*) c->base) + 8u * c->total + c->offset; }
static void set_id(Clusters* c, unsigned i, uint32_t v) { ((uint32_t*) c->base)[c->offset + i] = v; }
static void set_x(Clusters* c, unsigned i, float v) { ((float*) c->base)[c->total + 3 * (c->offset + i)] = v; }
static void set_y(Clusters* c, unsigned i, float v) { ((float*) c->base)[c->total + 3 * (c->offset + i) + 1] = v; }
static void set_z(Clusters* c, unsigned i, float v) { ((float*) c->base)[c->total + 3 * (c->offset + i) + 2] = v; }
static void set_phi(Clusters* c, unsigned i, int16_t v) { ((int16_t*) c->base)[8u * c->total + c->offset + i] = v; }

/* --------------------------------------------------------------------------------
 * phi (VeloTools.cuh:18-63, signselect BackendCommon.h:183)
 * ------------------------------------------------------------------------------ */
static float fast_atan2f(float y, float x)
{
  const float c1 = .25f * pi_f;
  const float c2 = .75f * pi_f;
  const float abs_y = fabsf(y);
  const float x_plus_y = x + abs_y;
  const float x_sub_y = x - abs_y;
  const float y_sub_x = abs_y - x;
  const float nom = (x > 0) ? x_sub_y : x_plus_y;
  const float den = (x > 0) ? x_plus_y : y_sub_x;
  const float r = nom / den;
  const float angle = ((x > 0) ? c1 : c2) - c1 * r;
  return copysignf(angle, y);
}

static float convert_factor_i16(void) { return 32768.f / pi_f; }

/* float -> int16 through a 32-bit truncation, as the reference's x86 build does */
static int16_t float_to_i16(float v) { return (int16_t) (int32_t) v; }

static int16_t hit_phi_16(float x, float y) { return float_to_i16(fast_atan2f(y, x) * convert_factor_i16()); }

/* BinarySearch.cuh:15-30 */
static int binary_search_leftmost(const int16_t* a, unsigned n, int16_t value)
{
  int l = 0, r = (int) n;
  while (l < r) {
    const int m = (l + r) / 2;
    if (value > a[m]) l = m + 1;
    else r = m;
  }
  return l;
}

/* VeloEventModel.cuh:192-196 (float multiply, then truncation) */
static unsigned track_offset(const unsigned* offsets_est, unsigned event)
{
  const unsigned o = offsets_est[event * N_MODULE_PAIRS];
  return (unsigned) ((float) o * tracks_per_cluster);
}

/* host/prefix_sum/src/HostPrefixSum.cpp:76-108: out[0] = 0, out[i + 1] = sum(in[0..i]) */
static unsigned prefix_sum(Result* r, const char* name, const unsigned* in, size_t n, unsigned** out_p)
{
  unsigned* out = make(r, name, (n + 1) * sizeof(unsigned));
  unsigned s = 0;
  out[0] = 0;
  for (size_t i = 0; i < n; ++i) {
    s += in[i];
    out[i + 1] = s;
  }
  if (out_p) *out_p = out;
  return s;
}

/* --------------------------------------------------------------------------------
 * SP lookup tables: host/velo/clustering/src/ClusteringCommon.cpp:6-104.
 * For each 8-bit pattern (bit = col * 4 + row), 8-connected groups seeded in
 * ascending bit order; pattern byte = centroid row | col << 2 per cluster,
 * shifted by 4 for the second, bit 3 set when there is a second cluster.
 * ------------------------------------------------------------------------------ */
static void sp_tables(uint8_t patterns[256], float fx[512], float fy[512])
{
  memset(patterns, 0, 256);
  memset(fx, 0, 512 * sizeof(float));
  memset(fy, 0, 512 * sizeof(float));
  for (unsigned sp = 0; sp < 256; ++sp) {
    unsigned left = sp;
    unsigned clu = 0;
    for (unsigned seed = 0; seed < 8; ++seed) {
      if (!(left & (1u << seed))) continue;
      unsigned group = 1u << seed, grown;
      do {
        grown = group;
        for (unsigned b = 0; b < 8; ++b) {
          if (!(left & (1u << b)) || (group & (1u << b))) continue;
          const int col = (int) (b / 4), row = (int) (b % 4);
          for (unsigned o = 0; o < 8; ++o) {
            if (!(group & (1u << o))) continue;
            const int ocol = (int) (o / 4), orow = (int) (o % 4);
            if (abs(ocol - col) <= 1 && abs(orow - row) <= 1) {
              group |= 1u << b;
              break;
            }
          }
        }
      } while (group != grown);
      left &= ~group;
      unsigned x = 0, y = 0, n = 0;
      for (unsigned b = 0; b < 8; ++b)
        if (group & (1u << b)) {
          x += b / 4;
          y += b % 4;
          ++n;
        }
      const uint32_t cx = x / n, cy = y / n;
      fx[2 * sp + clu] = (float) x / (float) n - (float) cx;
      fy[2 * sp + clu] = (float) y / (float) n - (float) cy;
      patterns[sp] |= (uint8_t) (((cx << 2) | cy) << (4 * clu));
      patterns[sp] |= (uint8_t) (clu << 3);
      ++clu;
    }
  }
}

/* --------------------------------------------------------------------------------
 * 1. velo_calculate_number_of_candidates (VeloCalculateNumberOfCandidates.cu:9-48)
 * ------------------------------------------------------------------------------ */
static void calculate_number_of_candidates(const VeloCpuInput* in, unsigned* n_candidates, unsigned* bank_index)
{
  const unsigned n = in->n_events;
  const unsigned grid = (n + 255) / 256;
  for (unsigned block = 0; block < grid; ++block) {
    for (unsigned e = block; e < n; e += grid) {
      const RawEvent ev = raw_event(in, e + in->event_start);
      unsigned count = 0;
      for (unsigned b = 0; b < ev.n_banks; ++b) {
        const RawBank bank = raw_bank(&ev, b, in->bank_version);
        if (is_velo_bank(&bank)) count += (in->bank_version == 2 || in->bank_version == 3) ? bank.count : bank.size / 4u;
        if (block == 0) {
          if (in->bank_version > 3) {
            bank_index[sensor_index0(&bank)] = b;
            bank_index[sensor_index1(&bank)] = b;
          }
          else {
            bank_index[sensor_pair(&bank)] = b;
          }
        }
      }
      n_candidates[e] = 2 * count;
    }
  }
}

/* --------------------------------------------------------------------------------
 * 2. velo_estimate_input_size (EstimateInputSize.cu:9-239)
 * ------------------------------------------------------------------------------ */
static unsigned clz32(uint32_t v) { return v ? (unsigned) __builtin_clz(v) : 32u; }

static void estimate_bank(
  unsigned* estimated, uint32_t* candidates, unsigned* candidate_num, const RawBank* bank, int version)
{
  const bool v23 = version == 2 || version == 3;
  unsigned* mp_size = estimated + (v23 ? sensor_pair(bank) / 8 : sensor_index0(bank) / 8);
  const uint32_t n_sp = bank_n_sp(bank, version);
  unsigned found = 0;
  for (uint32_t sp_index = 0; sp_index < n_sp; ++sp_index) {
    const uint32_t sp_word = bank->word[sp_index];
    const uint32_t no_neighbours = sp_word & 0x80000000u;
    const uint32_t sp_addr = (sp_word & 0x007FFF00u) >> 8;
    const uint32_t sp = sp_word & 0xFFu;
    const uint32_t sensor_number = v23 ? sensor_pair(bank) : (sensor_index0(bank) | ((sp_word >> 23) & 0x1u));
    if (no_neighbours) {
      const bool pattern_0 = (sp & 0x88) && !(sp & 0x44) && (sp & 0x33);
      const bool pattern_1 = (sp & 0xCC) && !(sp & 0x22) && (sp & 0x11);
      *mp_size += (pattern_0 | pattern_1) ? 2u : 1u;
    }
    else {
      uint32_t pixels = (sp & 0x0Fu) | ((sp & 0xF0u) << 2);
      const uint32_t sp_row = sp_addr & 0x3Fu;
      const uint32_t sp_col = sp_addr >> 6;
      /* every super pixel of the bank is scanned: the reference tests this SP's own
       * no-neighbour bit (always 0 here) instead of the other one's (line 113) */
      for (uint32_t k = 0; k < n_sp; ++k) {
        const uint32_t other_word = bank->word[k];
        const uint32_t other_addr = (other_word & 0x007FFF00u) >> 8;
        const uint32_t other_row = other_addr & 0x3Fu;
        const uint32_t other_col = other_addr >> 6;
        const uint32_t other_sp = other_word & 0xFFu;
        const bool is_top = other_row == (sp_row + 1) && other_col == sp_col;
        const bool is_top_right = other_row == (sp_row + 1) && other_col == (sp_col + 1);
        const bool is_right = other_row == sp_row && other_col == (sp_col + 1);
        const bool is_right_bottom = other_row == (sp_row - 1) && other_col == (sp_col + 1);
        const bool is_bottom = other_row == (sp_row - 1) && other_col == sp_col;
        if (is_top) pixels |= (((other_sp & 0x01u) | ((other_sp & 0x10u) << 2)) << 4);
        if (is_top_right) pixels |= ((other_sp & 0x01u) << 16);
        if (is_right) pixels |= ((other_sp & 0x0Fu) << 12);
        if (is_right_bottom) pixels |= ((other_sp & 0x08u) << 8);
        if (is_bottom) pixels |= ((other_sp & 0x80u) >> 2);
      }
      const uint32_t inside = pixels & 0x3CFu;
      const uint32_t mask = (inside << 1) | (inside << 5) | (inside << 6) | (inside << 7);
      const uint32_t working = mask & (~pixels);
      const uint32_t cand_tmp = (working >> 1) & (working >> 5) & (working >> 6) & (working >> 7);
      const uint32_t cands = cand_tmp & pixels;
      const uint32_t consolidated = (cands & 0x0Fu) | ((cands >> 2) & 0xF0u);
      const uint32_t first = consolidated & 0x33u;
      const uint32_t second = consolidated & 0xCCu;
      if (first) {
        candidates[(*candidate_num)++] = (sp_index << 11) | (sensor_number << 3) | (clz32(first) - 24);
        ++found;
      }
      if (second) {
        candidates[(*candidate_num)++] = (sp_index << 11) | (sensor_number << 3) | (clz32(second) - 24);
        ++found;
      }
    }
  }
  if (found > 0) *mp_size += found;
}

static void estimate_input_size(
  const VeloCpuInput* in,
  const unsigned* candidates_offsets,
  unsigned* estimated,
  unsigned* candidate_num,
  uint32_t* candidates)
{
  for (unsigned e = 0; e < in->n_events; ++e) {
    const RawEvent ev = raw_event(in, e + in->event_start);
    for (unsigned b = 0; b < ev.n_banks; ++b) {
      const RawBank bank = raw_bank(&ev, b, in->bank_version);
      if (!is_velo_bank(&bank)) continue;
      estimate_bank(
        estimated + e * N_MODULE_PAIRS, candidates + candidates_offsets[e], candidate_num + e, &bank, in->bank_version);
    }
  }
}

/* --------------------------------------------------------------------------------
 * 3. velo_masked_clustering (MaskedVeloClustering.cu:21-84, 131-576)
 * ------------------------------------------------------------------------------ */
static uint64_t make_8con_mask(uint64_t c)
{
  return c | ((c & 0x7FFF7FFF7FFF7FFFull) << 1) | ((c & 0xFFFEFFFEFFFEFFFEull) << 15) | (c << 16) |
         ((c & 0xFFFCFFFCFFFCFFFCull) << 17) | ((c & 0xFFFEFFFEFFFEFFFEull) >> 1) |
         ((c & 0x7FFF7FFF7FFF7FFFull) >> 15) | (c >> 16) | ((c & 0x3FFF3FFF3FFF3FFFull) >> 17);
}
static uint64_t mask_east(uint64_t c)
{
  const uint64_t m = c >> 48;
  return m | ((m & 0x7FFF7FFF7FFF7FFFull) << 1) | (m >> 1);
}
static uint64_t mask_west(uint64_t c)
{
  const uint64_t m = c << 48;
  return m | (m << 1) | ((m & 0xFFFEFFFEFFFEFFFEull) >> 1);
}
static unsigned popc64(uint64_t v) { return (unsigned) __builtin_popcountll(v); }

typedef struct {
  uint64_t pixels;
  uint32_t x, y, n;
} Cluster;

static Cluster make_cluster(uint64_t map, uint64_t start, uint32_t col_lower, uint32_t row_lower)
{
  uint64_t cur = 0, next = start;
  while (cur != next) {
    cur = next;
    next = map & make_8con_mask(cur);
  }
  Cluster c;
  c.pixels = cur;
  c.n = popc64(cur);
  c.x = col_lower * c.n + popc64(cur & 0x00000000FFFF0000ull) + popc64(cur & 0x0000FFFF00000000ull) * 2 +
        popc64(cur & 0xFFFF000000000000ull) * 3;
  uint32_t y = row_lower * c.n;
  for (unsigned r = 1; r <= 14; ++r)
    y += popc64(cur & (0x0001000100010001ull << r)) * r;
  c.y = y;
  return c;
}

static void store_cluster(Clusters* cont, unsigned index, uint32_t cid, float gx, float gy, float gz)
{
  set_id(cont, index, lhcb_id(cid));
  set_x(cont, index, gx);
  set_y(cont, index, gy);
  set_z(cont, index, gz);
  set_phi(cont, index, hit_phi_16(gx, gy));
}

static void no_neighbour_sp(
  const Geometry* g,
  const uint8_t* patterns,
  const float* sp_fx,
  const float* sp_fy,
  Clusters* cont,
  unsigned* mp_cluster_num,
  unsigned module_pair,
  unsigned cluster_start,
  const RawBank* bank,
  int version)
{
  const bool v23 = version == 2 || version == 3;
  const float* ltg0 = g->ltg + 12 * (v23 ? sensor_pair(bank) : sensor_index0(bank));
  const float* ltg1 = g->ltg + 12 * sensor_index1(bank);
  const uint32_t n_sp = bank_n_sp(bank, version);
  for (uint32_t i = 0; i < n_sp; ++i) {
    const uint32_t sp_word = bank->word[i];
    if (!(sp_word & 0x80000000u)) continue;
    const uint32_t sp_addr = (sp_word & 0x007FFF00u) >> 8;
    const bool bit23 = (sp_word & 0x800000u) != 0;
    /* v2/v3 use the unmasked sourceID for the channel id but the masked one for ltg */
    const uint32_t sensor_index = v23 ? bank->source_id : (bit23 ? sensor_index1(bank) : sensor_index0(bank));
    const float* ltg = (!v23 && bit23) ? ltg1 : ltg0;
    const int32_t sp_row = (int32_t) (sp_addr & 0x3Fu);
    const int32_t sp_col = (int32_t) (sp_addr >> 6);
    const uint32_t sp = sp_word & 0xFFu;
    const uint32_t idx = patterns[sp];
    const uint32_t chip = (uint32_t) sp_col >> 7;
    for (unsigned k = 0; k < 2; ++k) {
      if (k == 1 && !(idx & 8)) break;
      const uint32_t row = k ? (idx >> 4) & 3u : idx & 3u;
      const uint32_t col = k ? (idx >> 6) & 1u : (idx >> 2) & 1u;
      const uint32_t cx = (uint32_t) sp_col * 2 + col;
      const uint32_t cy = (uint32_t) sp_row * 4 + row;
      const uint32_t cid = channel_id(sensor_index, chip, cx & 0xFFu, cy);
      const float fx = sp_fx[sp * 2 + k];
      const float fy = sp_fy[sp * 2 + k];
      const float local_x = g->local_x[cx] + fx * g->x_pitch[cx];
      const float local_y = ((float) cy + 0.5f + fy) * pixel_size;
      const unsigned num = mp_cluster_num[module_pair]++;
      const float gx = ltg[0] * local_x + ltg[1] * local_y + ltg[9];
      const float gy = ltg[3] * local_x + ltg[4] * local_y + ltg[10];
      const float gz = ltg[6] * local_x + ltg[7] * local_y + ltg[11];
      store_cluster(cont, cluster_start + num, cid, gx, gy, gz);
    }
  }
}

static void rest_of_clusters(
  const Geometry* g,
  const unsigned* mp_cluster_start,
  Clusters* cont,
  unsigned* mp_cluster_num,
  uint32_t candidate,
  const RawBank* bank,
  int version)
{
  const uint32_t sp_index = candidate >> 11;
  const uint32_t sensor_number = (candidate >> 3) & 0xFFu;
  const uint32_t module_pair = sensor_number / 8;
  const uint32_t start_loc = candidate & 0x7u;
  const float* ltg = g->ltg + 12 * sensor_number;
  const uint32_t n_sp = bank_n_sp(bank, version);

  const uint32_t sp_word = bank->word[sp_index];
  const uint32_t sp_addr = (sp_word & 0x007FFF00u) >> 8;
  const int32_t sp_row = (int32_t) (sp_addr & 0x3Fu);
  const int32_t sp_col = (int32_t) (sp_addr >> 6);

  uint32_t pa[5] = {0, 0, 0, 0, 0};
  const int32_t r_lo = sp_row - 2, r_hi = sp_row + 1;
  const int32_t c_lo = sp_col - 3, c_hi = sp_col + 1;
  const int32_t row_lower = r_lo * 4;
  const int32_t col_lower = c_lo * 2;

  for (uint32_t k = 0; k < n_sp; ++k) {
    const uint32_t ow = bank->word[k];
    if (version > 3) {
      const uint32_t other_bit = (ow & 0x800000u) ? 1u : 0u;
      if (other_bit != (sensor_number & 0x1u)) continue;
    }
    if (ow & 0x80000000u) continue;
    const uint32_t oaddr = (ow & 0x007FFF00u) >> 8;
    const int32_t orow = (int32_t) (oaddr & 0x3Fu);
    const int32_t ocol = (int32_t) (oaddr >> 6);
    const uint32_t osp = ow & 0xFFu;
    if (orow >= r_lo && orow <= r_hi && ocol >= c_lo && ocol <= c_hi) {
      const int rel_row = orow - r_lo;
      const int rel_col = ocol - c_lo;
      pa[rel_col] |= ((osp & 0x0Fu) << (4 * rel_row)) | ((osp & 0xF0u) << (12 + 4 * rel_row));
    }
  }

  const uint32_t rel_row0 = start_loc & 0x3u;
  const uint32_t rel_col0 = start_loc < 4 ? 1u : 0u;
  const uint32_t col = (uint32_t) sp_col * 2 + rel_col0;
  const uint64_t start = ((uint64_t) (0x01u << (11 - rel_row0)) << (16 * (col & 0x01u))) << 32;
  const uint64_t map = (((uint64_t) pa[3]) << 32) | pa[2];
  const Cluster cl = make_cluster(map, start, (uint32_t) (col_lower + 4), (uint32_t) row_lower);

  const uint64_t precedence = (mask_east(cl.pixels) & pa[4]) | (cl.pixels & (start ^ (0 - start)));
  bool keep = precedence == 0 && !popc64(cl.pixels & 0x8000800080008000ull) &&
              !popc64(cl.pixels & 0x0001000100010001ull);
  if (!keep) return;
  uint32_t x = cl.x, y = cl.y, n = cl.n;
  if (popc64(cl.pixels & 0xFFFFull)) {
    const uint64_t west_map = (((uint64_t) pa[1]) << 32) | pa[0];
    const uint64_t west_start = mask_west(cl.pixels) & west_map;
    const Cluster ext = make_cluster(west_map, west_start, (uint32_t) col_lower, (uint32_t) row_lower);
    x += ext.x;
    y += ext.y;
    n += ext.n;
    keep = keep && !popc64(ext.pixels & 0x8000800080008000ull) && !popc64(ext.pixels & 0xFFFFull) &&
           !popc64(cl.pixels & 0x0001000100010001ull);
  }
  if (!keep) return;
  /* A candidate whose bank index names another bank (a slice with more than one bank per
   * sensor, e.g. VP and VPRetinaCluster banks together) can leave the start pixel outside the
   * map: no pixel, and the reference divides by zero (MaskedVeloClustering.cu:461-462); the
   * candidate makes no cluster here, as on the GPU. */
  if (n == 0) return;
  const uint32_t cx = x / n;
  const uint32_t cy = y / n;
  const float fx = (float) x / (float) n - (float) cx;
  const float fy = (float) y / (float) n - (float) cy;
  const uint32_t chip = cx >> 8;
  const uint32_t cid = channel_id(sensor_number, chip, cx & 0xFFu, cy);
  const float local_x = g->local_x[cx] + fx * g->x_pitch[cx];
  const float local_y = ((float) cy + 0.5f + fy) * pixel_size;
  const unsigned num = mp_cluster_num[module_pair]++;
  const float gx = ltg[0] * local_x + ltg[1] * local_y + ltg[9];
  const float gy = ltg[3] * local_x + ltg[4] * local_y + ltg[10];
  const float gz = ltg[6] * local_x + ltg[7] * local_y + ltg[11];
  store_cluster(cont, mp_cluster_start[module_pair] + num, cid, gx, gy, gz);
}

static void masked_clustering(
  const VeloCpuInput* in,
  const Geometry* g,
  const uint8_t* patterns,
  const float* sp_fx,
  const float* sp_fy,
  const unsigned* offsets_est,
  const unsigned* candidate_num,
  const uint32_t* candidates,
  const unsigned* candidates_offsets,
  const unsigned* bank_index,
  unsigned* cluster_num,
  char* container)
{
  const unsigned n = in->n_events;
  Clusters cont = {container, offsets_est[N_MODULE_PAIRS * n], 0};
  const bool v23 = in->bank_version == 2 || in->bank_version == 3;
  for (unsigned e = 0; e < n; ++e) {
    const unsigned* mp_start = offsets_est + e * N_MODULE_PAIRS;
    unsigned* mp_num = cluster_num + e * N_MODULE_PAIRS;
    const RawEvent ev = raw_event(in, e + in->event_start);
    for (unsigned b = 0; b < ev.n_banks; ++b) {
      const RawBank bank = raw_bank(&ev, b, in->bank_version);
      if (!is_velo_bank(&bank)) continue;
      const unsigned mp = v23 ? sensor_pair(&bank) / 8 : sensor_index0(&bank) / 8;
      no_neighbour_sp(g, patterns, sp_fx, sp_fy, &cont, mp_num, mp, mp_start[mp], &bank, in->bank_version);
    }
    const uint32_t* cands = candidates + candidates_offsets[e];
    for (unsigned c = 0; c < candidate_num[e]; ++c) {
      const uint32_t sensor = (cands[c] >> 3) & 0xFFu;
      const RawBank bank = raw_bank(&ev, bank_index[sensor], in->bank_version);
      rest_of_clusters(g, mp_start, &cont, mp_num, cands[c], &bank, in->bank_version);
    }
  }
}

/* --------------------------------------------------------------------------------
 * 4. velo_sort_by_phi (SortByPhi.cu:49-153): rank by (phi, id) inside each module
 *    pair, then gather over the event's whole estimated range; slots of the
 *    estimate that hold no cluster keep permutation 0 (the memset value).
 * ------------------------------------------------------------------------------ */
static void sort_by_phi(
  unsigned n,
  const unsigned* offsets_est,
  const unsigned* cluster_num,
  char* container,
  char* sorted,
  unsigned* perm)
{
  const unsigned total = offsets_est[N_MODULE_PAIRS * n];
  Clusters in = {container, total, 0};
  Clusters out = {sorted, total, 0};
  for (unsigned e = 0; e < n; ++e) {
    const unsigned* start = offsets_est + e * N_MODULE_PAIRS;
    const unsigned* num = cluster_num + e * N_MODULE_PAIRS;
    for (unsigned mp = 0; mp < N_MODULE_PAIRS; ++mp) {
      for (unsigned i = 0; i < num[mp]; ++i) {
        const unsigned hi = start[mp] + i;
        const int16_t phi = c_phi(&in, hi);
        unsigned position = 0;
        for (unsigned j = 0; j < num[mp]; ++j) {
          const unsigned hj = start[mp] + j;
          const int16_t other = c_phi(&in, hj);
          position += phi > other || (hi != hj && phi == other && c_id(&in, hi) > c_id(&in, hj));
        }
        perm[start[mp] + position] = hi;
      }
    }
    const unsigned first = start[0];
    const unsigned count = start[N_MODULE_PAIRS] - first;
    for (unsigned i = 0; i < count; ++i) {
      const unsigned src = perm[first + i];
      set_id(&out, first + i, c_id(&in, src));
      set_phi(&out, first + i, c_phi(&in, src));
      set_x(&out, first + i, c_x(&in, src));
      set_y(&out, first + i, c_y(&in, src));
      set_z(&out, first + i, c_z(&in, src));
    }
  }
}

/* --------------------------------------------------------------------------------
 * 5. velo_search_by_triplet (SearchByTriplet.cu:110-609; scalar seeding, the
 *    dispatch the reference takes with ALWAYS_DISPATCH_TO_DEFAULT)
 * ------------------------------------------------------------------------------ */
typedef struct {
  uint16_t hits[MAX_TRACK_SIZE];
  uint8_t hitsNum;
  uint8_t pad;
} TrackHits; /* 54 bytes, as Velo::TrackHits */
typedef struct {
  uint16_t hits[3];
} TrackletHits;

typedef struct {
  unsigned hit_start;
  unsigned hit_num;
  float z[2];
} ModulePair;

enum { ATOMIC_THREE_HIT = 0, ATOMIC_TTF = 1, ATOMIC_LOCAL_HITS = 2 };
#define BIT_SEED 0x80000000u
#define BIT_TRACK_NUMBER 0x0FFFFFFFu
#define BIT_SKIPPED 0x70000000u

typedef struct {
  Clusters hits;
  const int16_t* phi;
  bool* used;
  uint16_t* h1_indices;
  TrackletHits* tracklets;
  unsigned* ttf;
  TrackHits* tracks;
  TrackletHits* three_hit;
  unsigned* atomics;
  unsigned* n_tracks;
  float max_scatter;
  int16_t phi_tol;
  unsigned max_skipped;
  ModulePair md[3];
} SearchState;

typedef struct {
  int16_t candidate;
  int16_t phi;
} Forward;

static Forward find_forward_candidate(
  const ModulePair* mp, const int16_t* phis, float h0x, float h0y, float tx, float ty, float dz, int16_t tol)
{
  const float predx = tx * dz;
  const float predy = ty * dz;
  const float xp = h0x + predx;
  const float yp = h0y + predy;
  Forward f;
  f.phi = hit_phi_16(xp, yp);
  f.candidate = (int16_t) binary_search_leftmost(phis + mp->hit_start, mp->hit_num, (int16_t) (f.phi - tol));
  return f;
}

static void track_seeding(SearchState* s, unsigned candidates_to_consider)
{
  const ModulePair* prev = &s->md[0];
  const ModulePair* cur = &s->md[1];
  const ModulePair* next = &s->md[2];
  for (unsigned r = 0; r < cur->hit_num; ++r) {
    const unsigned h1 = cur->hit_start + r;
    if (!s->used[h1]) s->h1_indices[s->atomics[ATOMIC_LOCAL_HITS]++] = (uint16_t) h1;
  }
  const unsigned n_h1 = s->atomics[ATOMIC_LOCAL_HITS];
  for (unsigned r = 0; r < n_h1; ++r) {
    const uint16_t h1 = s->h1_indices[r];
    uint16_t best_h0 = 0, best_h2 = 0;
    float best_fit = s->max_scatter;
    const float h1x = c_x(&s->hits, h1), h1y = c_y(&s->hits, h1), h1z = c_z(&s->hits, h1);
    const int16_t h1_phi = c_phi(&s->hits, h1);
    unsigned best_h0s[8];
    int phi_index = binary_search_leftmost(s->phi + prev->hit_start, prev->hit_num, h1_phi);
    unsigned found = 0;
    for (unsigned i = 0; i < prev->hit_num && found < candidates_to_consider; ++i) {
      const int diff = (i & 1u) ? (int) i : -(int) i;
      phi_index += diff;
      const unsigned in_bounds =
        phi_index < 0 ? (unsigned) phi_index + prev->hit_num :
                        (phi_index >= (int) prev->hit_num ? (unsigned) (phi_index - (int) prev->hit_num) :
                                                            (unsigned) phi_index);
      const unsigned h0 = prev->hit_start + in_bounds;
      if (!s->used[h0]) best_h0s[found++] = h0;
    }
    for (unsigned c = 0; c < found; ++c) {
      const unsigned h0 = best_h0s[c];
      const float h0x = c_x(&s->hits, h0), h0y = c_y(&s->hits, h0), h0z = c_z(&s->hits, h0);
      const float td = 1.0f / (h1z - h0z);
      const float txn = h1x - h0x;
      const float tyn = h1y - h0y;
      const float tx = txn * td;
      const float ty = tyn * td;
      const Forward f =
        find_forward_candidate(next, s->phi, h0x, h0y, tx, ty, next->z[0] - prev->z[0], s->phi_tol);
      for (unsigned i = 0; i < next->hit_num; ++i) {
        const unsigned in_bounds = ((unsigned) (int) f.candidate + i) % next->hit_num;
        const unsigned h2 = next->hit_start + in_bounds;
        const int16_t phi_diff = (int16_t) (c_phi(&s->hits, h2) - f.phi);
        const int16_t abs_diff = (int16_t) (phi_diff < 0 ? -phi_diff : phi_diff);
        if (abs_diff > s->phi_tol) break;
        if (!s->used[h2]) {
          const float dz = c_z(&s->hits, h2) - h0z;
          const float predx = h0x + tx * dz;
          const float predy = h0y + ty * dz;
          const float dx = predx - c_x(&s->hits, h2);
          const float dy = predy - c_y(&s->hits, h2);
          const float scatter = dx * dx + dy * dy;
          if (scatter < best_fit) {
            best_fit = scatter;
            best_h0 = (uint16_t) h0;
            best_h2 = (uint16_t) h2;
          }
        }
      }
    }
    if (best_fit < s->max_scatter) {
      const unsigned tn = s->atomics[ATOMIC_TTF]++ % MAX_TTF;
      s->tracklets[tn].hits[0] = best_h0;
      s->tracklets[tn].hits[1] = h1;
      s->tracklets[tn].hits[2] = best_h2;
      s->ttf[tn] = BIT_SEED | tn;
    }
  }
}

static void track_forwarding(SearchState* s, unsigned diff_ttf, unsigned prev_ttf, unsigned event)
{
  const ModulePair* next = &s->md[2];
  for (unsigned k = 0; k < diff_ttf; ++k) {
    const unsigned full = s->ttf[(prev_ttf + k) % MAX_TTF];
    const bool is_seed = (full & BIT_SEED) == BIT_SEED;
    const unsigned skipped = (full & BIT_SKIPPED) >> 28;
    unsigned tn = full & BIT_TRACK_NUMBER;
    /* a seed is read through the same view as a track: only hits[0..2] are touched */
    uint16_t* thits;
    unsigned nh;
    uint8_t* thits_num = NULL;
    if (is_seed) {
      thits = s->tracklets[tn].hits;
      nh = 3;
    }
    else {
      thits = s->tracks[tn].hits;
      thits_num = &s->tracks[tn].hitsNum;
      nh = *thits_num;
    }
    const uint16_t h0 = thits[nh - 2];
    const uint16_t h1 = thits[nh - 1];
    const float h0x = c_x(&s->hits, h0), h0y = c_y(&s->hits, h0), h0z = c_z(&s->hits, h0);
    const unsigned h0_module = ((c_id(&s->hits, h0) & 0x3FC0000u) >> 18) / 4;
    const float h1x = c_x(&s->hits, h1), h1y = c_y(&s->hits, h1), h1z = c_z(&s->hits, h1);
    const float td = 1.0f / (h1z - h0z);
    const float txn = h1x - h0x;
    const float tyn = h1y - h0y;
    const float tx = txn * td;
    const float ty = tyn * td;
    float best_fit = s->max_scatter;
    int best_h2 = -1;
    const Forward f =
      find_forward_candidate(next, s->phi, h0x, h0y, tx, ty, next->z[h0_module % 2] - h0z, s->phi_tol);
    for (unsigned i = 0; i < next->hit_num; ++i) {
      const unsigned in_bounds = ((unsigned) (int) f.candidate + i) % next->hit_num;
      const unsigned h2 = next->hit_start + in_bounds;
      const int16_t phi_diff = (int16_t) (c_phi(&s->hits, h2) - f.phi);
      const int16_t abs_diff = (int16_t) (phi_diff < 0 ? -phi_diff : phi_diff);
      if (abs_diff > s->phi_tol) break;
      const float dz = c_z(&s->hits, h2) - h0z;
      const float predx = h0x + tx * dz;
      const float predy = h0y + ty * dz;
      const float dx = predx - c_x(&s->hits, h2);
      const float dy = predy - c_y(&s->hits, h2);
      const float scatter = dx * dx + dy * dy;
      if (scatter < best_fit) {
        best_fit = scatter;
        best_h2 = (int) h2;
      }
    }
    if (best_h2 != -1) {
      s->used[best_h2] = true;
      if (nh == 3) {
        s->used[thits[0]] = true;
        s->used[thits[1]] = true;
        s->used[thits[2]] = true;
        tn = s->n_tracks[event]++;
        s->tracks[tn].hits[0] = thits[0];
        s->tracks[tn].hits[1] = thits[1];
        s->tracks[tn].hits[2] = thits[2];
        s->tracks[tn].hits[3] = (uint16_t) best_h2;
        s->tracks[tn].hitsNum = 4;
      }
      else {
        thits[(*thits_num)++] = (uint16_t) best_h2;
      }
      if (nh + 1 < MAX_TRACK_SIZE) s->ttf[s->atomics[ATOMIC_TTF]++ % MAX_TTF] = tn;
    }
    else if (skipped < s->max_skipped) {
      const unsigned requeued = ((skipped + 1) << 28) | (full & (BIT_SEED | BIT_TRACK_NUMBER));
      s->ttf[s->atomics[ATOMIC_TTF]++ % MAX_TTF] = requeued;
    }
    else if (nh == 3) {
      TrackletHits* t3 = &s->three_hit[s->atomics[ATOMIC_THREE_HIT]++];
      t3->hits[0] = thits[0];
      t3->hits[1] = thits[1];
      t3->hits[2] = thits[2];
    }
  }
}

static void load_module_pairs(SearchState* s, unsigned first, const unsigned* start, const unsigned* num, unsigned hit_offset, const Geometry* g)
{
  for (unsigned i = 0; i < 3; ++i) {
    const unsigned mp = first - i;
    s->md[i].hit_start = start[mp] - hit_offset;
    s->md[i].hit_num = num[mp];
    s->md[i].z[0] = g->module_zs[2 * mp];
    s->md[i].z[1] = g->module_zs[2 * mp + 1];
  }
}

static void search_by_triplet(
  const VeloCpuInput* in,
  const Geometry* g,
  const unsigned* offsets_est,
  const unsigned* cluster_num,
  char* sorted,
  TrackHits* tracks,
  TrackletHits* tracklets,
  unsigned* ttf,
  TrackletHits* three_hit,
  bool* hit_used,
  unsigned* atomics,
  uint16_t* rel_indices,
  unsigned* n_tracks)
{
  const unsigned n = in->n_events;
  const unsigned total = offsets_est[N_MODULE_PAIRS * n];
  for (unsigned e = 0; e < n; ++e) {
    const unsigned* start = offsets_est + e * N_MODULE_PAIRS;
    const unsigned* num = cluster_num + e * N_MODULE_PAIRS;
    const unsigned hit_offset = start[0];
    SearchState s;
    s.hits.base = sorted;
    s.hits.total = total;
    s.hits.offset = hit_offset;
    s.phi = c_phi_begin(&s.hits);
    s.used = hit_used + hit_offset;
    s.h1_indices = rel_indices + hit_offset;
    s.tracklets = tracklets + e * MAX_TTF;
    s.ttf = ttf + e * MAX_TTF;
    s.tracks = tracks + track_offset(offsets_est, e);
    s.three_hit = three_hit + track_offset(offsets_est, e);
    s.atomics = atomics + e * 3;
    s.n_tracks = n_tracks;
    s.max_scatter = in->max_scatter;
    s.phi_tol = float_to_i16(in->phi_tolerance * convert_factor_i16());
    s.max_skipped = in->max_skipped_modules;

    unsigned first = N_MODULE_PAIRS - 1;
    load_module_pairs(&s, first, start, num, hit_offset, g);
    track_seeding(&s, 8);
    unsigned last_ttf = 0;
    --first;
    while (first > 1) {
      load_module_pairs(&s, first, start, num, hit_offset, g);
      const unsigned prev_ttf = last_ttf;
      last_ttf = s.atomics[ATOMIC_TTF];
      const unsigned diff = last_ttf - prev_ttf;
      s.atomics[ATOMIC_LOCAL_HITS] = 0;
      track_forwarding(&s, diff, prev_ttf, e);
      track_seeding(&s, 4);
      --first;
    }
    const unsigned prev_ttf = last_ttf;
    last_ttf = s.atomics[ATOMIC_TTF];
    const unsigned diff = last_ttf - prev_ttf;
    for (unsigned k = 0; k < diff; ++k) {
      const unsigned full = s.ttf[(prev_ttf + k) % MAX_TTF];
      if ((full & BIT_SEED) == BIT_SEED) {
        const TrackletHits* t = &s.tracklets[full & BIT_TRACK_NUMBER];
        s.three_hit[s.atomics[ATOMIC_THREE_HIT]++] = *t;
      }
    }
  }
}

/* --------------------------------------------------------------------------------
 * 6. velo_three_hit_tracks_filter (ThreeHitTracksFilter.cu:48-169)
 * ------------------------------------------------------------------------------ */
static float means_square_fit_chi2(const Clusters* c, const TrackletHits* t)
{
  float s0, sx, sz, sxz, sz2, u0, uy, uz, uyz, uz2;
  s0 = sx = sz = sxz = sz2 = 0.0f;
  u0 = uy = uz = uyz = uz2 = 0.0f;
  for (unsigned h = 0; h < 3; ++h) {
    const unsigned hn = t->hits[h];
    const float x = c_x(c, hn), y = c_y(c, hn), z = c_z(c, hn);
    const float wx = param_w, wx_t_x = wx * x, wx_t_z = wx * z;
    s0 += wx;
    sx += wx_t_x;
    sz += wx_t_z;
    sxz += wx_t_x * z;
    sz2 += wx_t_z * z;
    const float wy = param_w, wy_t_y = wy * y, wy_t_z = wy * z;
    u0 += wy;
    uy += wy_t_y;
    uz += wy_t_z;
    uyz += wy_t_y * z;
    uz2 += wy_t_z * z;
  }
  const float dens = 1.0f / (sz2 * s0 - sz * sz);
  const float state_tx = (sxz * s0 - sx * sz) * dens;
  const float state_x = (sx * sz2 - sxz * sz) * dens;
  const float denu = 1.0f / (uz2 * u0 - uz * uz);
  const float state_ty = (uyz * u0 - uy * uz) * denu;
  const float state_y = (uy * uz2 - uyz * uz) * denu;
  float chi2 = 0.0f;
  for (unsigned h = 0; h < 3; ++h) {
    const unsigned hn = t->hits[h];
    const float z = c_z(c, hn);
    const float x = state_x + state_tx * z;
    const float y = state_y + state_ty * z;
    const float dx = x - c_x(c, hn);
    const float dy = y - c_y(c, hn);
    chi2 += dx * dx * param_w + dy * dy * param_w;
  }
  return chi2 * 0.5f;
}

static void three_hit_tracks_filter(
  const VeloCpuInput* in,
  const unsigned* offsets_est,
  char* sorted,
  const TrackletHits* three_in,
  const unsigned* atomics,
  const bool* hit_used,
  TrackletHits* three_out,
  unsigned* n_out)
{
  const unsigned n = in->n_events;
  const unsigned total = offsets_est[N_MODULE_PAIRS * n];
  for (unsigned e = 0; e < n; ++e) {
    const unsigned hit_offset = offsets_est[e * N_MODULE_PAIRS];
    const bool* used = hit_used + hit_offset;
    const Clusters c = {sorted, total, hit_offset};
    const unsigned to = track_offset(offsets_est, e);
    const unsigned n_in = atomics[e * 3 + ATOMIC_THREE_HIT];
    for (unsigned t = 0; t < n_in; ++t) {
      const TrackletHits* trk = &three_in[to + t];
      const bool any_used = used[trk->hits[0]] || used[trk->hits[1]] || used[trk->hits[2]];
      const float chi2 = means_square_fit_chi2(&c, trk);
      if (!any_used && chi2 < in->max_chi2) three_out[to + n_out[e]++] = *trk;
    }
  }
}

/* --------------------------------------------------------------------------------
 * 7. velo_copy_track_hit_number (VeloCopyTrackHitNumber.cu:49-78)
 * ------------------------------------------------------------------------------ */
static void copy_track_hit_number(
  unsigned n,
  const unsigned* offsets_est,
  const TrackHits* tracks,
  const unsigned* offsets_tracks,
  const unsigned* offsets_three,
  unsigned* hit_number,
  unsigned* offsets_all)
{
  for (unsigned e = 0; e < n; ++e) {
    const TrackHits* et = tracks + track_offset(offsets_est, e);
    const unsigned nt = offsets_tracks[e + 1] - offsets_tracks[e];
    const unsigned n3 = offsets_three[e + 1] - offsets_three[e];
    unsigned* out = hit_number + offsets_tracks[e] + offsets_three[e];
    for (unsigned i = 0; i < nt; ++i)
      out[i] = et[i].hitsNum;
    for (unsigned i = 0; i < n3; ++i)
      out[nt + i] = 3;
    offsets_all[e + 1] = offsets_tracks[e + 1] + offsets_three[e + 1];
  }
}

/* --------------------------------------------------------------------------------
 * 8. velo_consolidate_tracks (VeloConsolidateTracks.cu:120-192; ConsolidatedTypes.cuh:95-122)
 * ------------------------------------------------------------------------------ */
static void consolidate_tracks(
  unsigned n,
  const unsigned* offsets_est,
  const unsigned* offsets_all,
  const TrackHits* tracks,
  const unsigned* offsets_hit_number,
  char* sorted,
  const TrackletHits* three_out,
  const unsigned* offsets_three,
  char* track_hits)
{
  const unsigned total_est = offsets_est[N_MODULE_PAIRS * n];
  const unsigned total_hits = offsets_hit_number[offsets_all[n]];
  for (unsigned e = 0; e < n; ++e) {
    const unsigned to = track_offset(offsets_est, e);
    const TrackHits* et = tracks + to;
    const TrackletHits* e3 = three_out + to;
    const unsigned n_total = offsets_all[e + 1] - offsets_all[e];
    const unsigned n3 = offsets_three[e + 1] - offsets_three[e];
    const unsigned n_main = n_total - n3;
    const Clusters c = {sorted, total_est, offsets_est[e * N_MODULE_PAIRS]};
    for (unsigned i = 0; i < n_total; ++i) {
      Clusters out = {track_hits, total_hits, offsets_hit_number[offsets_all[e] + i]};
      const uint16_t* h = i < n_main ? et[i].hits : e3[i - n_main].hits;
      const unsigned nh = i < n_main ? et[i].hitsNum : 3u;
      for (unsigned j = 0; j < nh; ++j) {
        set_x(&out, j, c_x(&c, h[j]));
        set_y(&out, j, c_y(&c, h[j]));
        set_z(&out, j, c_z(&c, h[j]));
      }
      for (unsigned j = 0; j < nh; ++j)
        set_id(&out, j, c_id(&c, h[j]));
    }
  }
}

/* --------------------------------------------------------------------------------
 * The chain (velo_reconstruction.py:72-292), buffers sized as each
 * set_arguments_size does.
 * ------------------------------------------------------------------------------ */
/* --------------------------------------------------------------------------------
 * Retina-cluster decoding (VPRetinaCluster banks, type 73):
 * calculate_number_of_retinaclusters_each_sensor_pair (CalculateNumberOfRetinaClustersPerSensor.cu:12-48),
 * its prefix sum, and decode_retinaclusters (DecodeRetinaClusters.cu:11-383).
 * -------------------------------------------------------------------------------- */
static unsigned retina_sensors_per_event(int version) { return (version == 2 || version == 3) ? N_SENSORS : N_SENSORS / 2; }

/* CalculateNumberOfRetinaClustersPerSensor.cu:12-48; bank index written by the slice's first event */
static void retina_count(const VeloCpuInput* in, unsigned* pair_size, unsigned* bank_index)
{
  const int v = in->bank_version;
  const unsigned per_event = retina_sensors_per_event(v);
  for (unsigned e = 0; e < in->n_events; ++e) {
    const RawEvent ev = raw_event(in, in->event_start + e);
    unsigned* size = pair_size + (size_t) e * per_event;
    for (unsigned b = 0; b < ev.n_banks; ++b) {
      const RawBank bank = raw_bank(&ev, b, v);
      if (bank.type == 73) {
        if (v == 2 || v == 3) size[bank.source_id] = bank.count;
        else size[sensor_pair(&bank)] = bank.size / 4u;
      }
      if (e == 0) bank_index[sensor_pair(&bank)] = b;
    }
  }
}

/* BinarySearch.cuh:33-47 */
static int binary_search_rightmost(const unsigned* a, unsigned n, unsigned value)
{
  int l = 0, r = (int) n;
  while (l < r) {
    const int m = (l + r) / 2;
    if (a[m] > value) r = m;
    else l = m + 1;
  }
  return r - 1;
}

typedef struct {
  uint32_t id;
  float x, y, z;
  int16_t phi;
  unsigned sensor;
} RetinaCluster;

/* populate_retinacluster / populate_sorting_key (DecodeRetinaClusters.cu:80-160, 246-303) */
static RetinaCluster retina_cluster(const Geometry* g, int v, const RawBank* bank, uint32_t w)
{
  RetinaCluster c;
  unsigned sensor;
  if (v == 2 || v == 3) sensor = bank->source_id;
  else sensor = ((w >> 22) & 0x1u) ? sensor_index1(bank) : sensor_index0(bank);
  uint32_t cx, cy, or_fx, or_fy;
  float fx, fy;
  if (v == 2) {
    cx = (w >> 14) & 0x3FFu;
    fx = ((w >> 11) & 0x7u) / 8.f;
    cy = (w >> 3) & 0xFFu;
    fy = (w & 0x7FFu) / 8.f;
    or_fx = 0;
    or_fy = 0;
  }
  else {
    cx = (w >> 12) & 0x3FFu;
    fx = ((w >> 10) & 0x3u) / 4.f;
    cy = (w >> 2) & 0xFFu;
    fy = (w & 0x3FFu) / 4.f;
    or_fx = ((w >> 11) & 0x1u) | ((w >> 10) & 0x1u);
    or_fy = ((w >> 1) & 0x1u) | (w & 0x1u);
  }
  const float* ltg = g->ltg + 12u * sensor;
  const float local_x = g->local_x[cx] + fx * g->x_pitch[cx];
  const float local_y = (0.5f + fy) * pixel_size;
  c.x = ltg[0] * local_x + ltg[1] * local_y + ltg[9];
  c.y = ltg[3] * local_x + ltg[4] * local_y + ltg[10];
  c.z = ltg[6] * local_x + ltg[7] * local_y + ltg[11];
  c.id = lhcb_id((or_fx << 27) | (or_fy << 26) | channel_id(sensor, cx >> 8, cx & 0xFFu, cy));
  c.phi = hit_phi_16(c.x, c.y);
  c.sensor = sensor;
  return c;
}

static void decode_retinaclusters(
  const VeloCpuInput* in, const Geometry* g, const unsigned* pair_offsets, const unsigned* bank_index,
  unsigned* cluster_num, unsigned* offsets_mp, char* container, unsigned* permutations, int64_t* keys)
{
  const int v = in->bank_version;
  const unsigned n = in->n_events;
  const unsigned per_event = retina_sensors_per_event(v);
  const unsigned step = per_event / N_MODULE_PAIRS;
  const unsigned total = pair_offsets[(size_t) n * per_event];
  /* populate_module_pair_offsets_and_sizes (:11-35); offsets_mp[0] stays 0 */
  for (unsigned el = 0; el < n * N_MODULE_PAIRS; ++el)
    offsets_mp[el + 1] = pair_offsets[(el + 1) * step];
  unsigned* zero_num = calloc((size_t) n * N_MODULE_PAIRS + 1, sizeof(unsigned));
  /* velo_calculate_sorting_key (:162-244) */
  for (unsigned e = 0; e < n; ++e) {
    const RawEvent ev = raw_event(in, in->event_start + e);
    const unsigned* so = pair_offsets + (size_t) e * per_event;
    const unsigned first = so[0], count = so[per_event] - first;
    for (unsigned k = 0; k < count; ++k) {
      const unsigned sp = (unsigned) binary_search_rightmost(so, per_event, first + k);
      const RawBank bank = raw_bank(&ev, bank_index[sp], v);
      if (bank.type != 73) continue;
      const uint32_t w = bank.word[k - (so[sp] - first)];
      const RetinaCluster c = retina_cluster(g, v, &bank, w);
      if (w != 0) ++cluster_num[e * N_MODULE_PAIRS + c.sensor / 8];
      else ++zero_num[e * N_MODULE_PAIRS + c.sensor / 8];
      keys[first + k] = w != 0 ? (int64_t) (((uint64_t) (uint16_t) c.phi << 48) | c.id) : INT64_MAX;
    }
  }
  /* velo_calculate_permutations (:37-78): rank by key among the module pair's entries */
  for (unsigned e = 0; e < n; ++e)
    for (unsigned mp = 0; mp < N_MODULE_PAIRS; ++mp) {
      const unsigned start = offsets_mp[e * N_MODULE_PAIRS + mp];
      const unsigned num = cluster_num[e * N_MODULE_PAIRS + mp] + zero_num[e * N_MODULE_PAIRS + mp];
      for (unsigned i = 0; i < num; ++i) {
        unsigned position = 0;
        for (unsigned j = 0; j < num; ++j)
          if (j != i) position += keys[start + i] > keys[start + j];
        permutations[start + i] = start + position;
      }
    }
  free(zero_num);
  /* decode_retinaclusters_sorted (:305-383) */
  Clusters out = {container, total, 0};
  for (unsigned e = 0; e < n; ++e) {
    const RawEvent ev = raw_event(in, in->event_start + e);
    const unsigned* so = pair_offsets + (size_t) e * per_event;
    const unsigned first = so[0], count = so[per_event] - first;
    for (unsigned k = 0; k < count; ++k) {
      const unsigned cn = first + k;
      const unsigned sp = (unsigned) binary_search_rightmost(so, per_event, cn);
      const RawBank bank = raw_bank(&ev, bank_index[sp], v);
      if (bank.type != 73) continue;
      const RetinaCluster c = retina_cluster(g, v, &bank, bank.word[cn - so[sp]]);
      const unsigned dst = permutations[cn];
      set_id(&out, dst, c.id);
      set_x(&out, dst, c.x);
      set_y(&out, dst, c.y);
      set_z(&out, dst, c.z);
      set_phi(&out, dst, c.phi);
    }
  }
}

/* --------------------------------------------------------------------------------
 * velo_kalman_filter (device/velo/simplified_kalman_filter/src/VeloKalmanFilter.cu:271-399,
 * include/VeloKalmanFilter.cuh:24-158), one track after the other.  Track hits are read from
 * the consolidated container (VeloConsolidated.cuh:19-88: ids, then x y z interleaved).
 * States go to Velo::Consolidated::States (VeloConsolidated.cuh:388-598): per track
 * x y z tx ty qop, then for all tracks c00 c20 c22 c11 c31 c33 chi2 ndof; qop, chi2 and
 * ndof are not written by the filter.
 * -------------------------------------------------------------------------------- */
typedef struct {
  float x, y, z, tx, ty, c00, c20, c22, c11, c31, c33;
} KalmanState;

static const float param_w_inverted = 0.00015625f; /* VeloDefinitions.cuh:36 */
static const float z_end_velo = 770.f;             /* VeloDefinitions.cuh:20 */

/* VeloKalmanFilter.cuh:24-58 */
static void kalman_step(float z, float zhit, float xhit, float whit, float* x, float* tx, float* cov_xx, float* cov_xtx, float* cov_txtx)
{
  const float dz = zhit - z;
  const float predx = *x + dz * *tx;
  const float dz_t_covTxTx = dz * *cov_txtx;
  const float predcovXTx = *cov_xtx + dz_t_covTxTx;
  const float dx_t_covXTx = dz * *cov_xtx;
  const float predcovXX = *cov_xx + 2.f * dx_t_covXTx + dz * dz_t_covTxTx;
  const float predcovTxTx = *cov_txtx;
  const float R = 1.0f / ((1.0f / whit) + predcovXX);
  const float Kx = predcovXX * R;
  const float KTx = predcovXTx * R;
  const float r = xhit - predx;
  *x = predx + Kx * r;
  *tx = *tx + KTx * r;
  *cov_xx = (1.f - Kx) * predcovXX;
  *cov_xtx = (1.f - Kx) * predcovXTx;
  *cov_txtx = predcovTxTx - KTx * predcovXTx;
}

typedef struct {
  const float* xyz; /* x y z of the track's first hit, 3 floats per hit */
  unsigned n;
} KalmanTrack;

/* VeloKalmanFilter.cuh:63-158 */
static KalmanState simplified_fit(const KalmanTrack* t, float state_tx, float state_ty, const float beamline[2], int backward, int upstream)
{
  const int direction = (backward ? 1 : -1) * (upstream ? 1 : -1);
  const float noise2PerLayer = 1e-8f + 7e-6f * (state_tx * state_tx + state_ty * state_ty);
  int firsthit = 0, lasthit = (int) t->n - 1, dhit = 1;
  if ((t->xyz[3 * lasthit + 2] - t->xyz[3 * firsthit + 2]) * (float) direction < 0) {
    const int temp = firsthit;
    firsthit = lasthit;
    lasthit = temp;
    dhit = -1;
  }
  KalmanState s;
  s.x = t->xyz[3 * firsthit];
  s.y = t->xyz[3 * firsthit + 1];
  s.z = t->xyz[3 * firsthit + 2];
  s.tx = state_tx;
  s.ty = state_ty;
  s.c00 = param_w_inverted;
  s.c11 = param_w_inverted;
  s.c20 = 0.f;
  s.c31 = 0.f;
  s.c22 = 1.f;
  s.c33 = 1.f;
  for (int i = firsthit + dhit; i != lasthit + dhit; i += dhit) {
    const float hx = t->xyz[3 * i], hy = t->xyz[3 * i + 1], hz = t->xyz[3 * i + 2];
    s.c22 += noise2PerLayer;
    s.c33 += noise2PerLayer;
    kalman_step(s.z, hz, hx, param_w, &s.x, &s.tx, &s.c00, &s.c20, &s.c22);
    kalman_step(s.z, hz, hy, param_w, &s.y, &s.ty, &s.c11, &s.c31, &s.c33);
    s.z = hz;
  }
  s.c22 += noise2PerLayer;
  s.c33 += noise2PerLayer;
  float delta_z;
  if (upstream)
    delta_z = (s.tx * (beamline[0] - s.x) + s.ty * (beamline[1] - s.y)) / (s.tx * s.tx + s.ty * s.ty);
  else
    delta_z = z_end_velo - s.z;
  s.x = s.x + s.tx * delta_z;
  s.y = s.y + s.ty * delta_z;
  s.z = s.z + delta_z;
  const float dz2 = delta_z * delta_z;
  s.c00 += dz2 * s.c22 + 2.f * delta_z * s.c20;
  s.c11 += dz2 * s.c33 + 2.f * delta_z * s.c31;
  s.c20 += s.c22 * delta_z;
  s.c31 += s.c33 * delta_z;
  return s;
}

static void store_state(float* base, unsigned total, unsigned i, const KalmanState* s)
{
  float* st = base + 6u * i;
  st[0] = s->x;
  st[1] = s->y;
  st[2] = s->z;
  st[3] = s->tx;
  st[4] = s->ty;
  float* cov = base + 6u * total + 8u * i;
  cov[0] = s->c00;
  cov[1] = s->c20;
  cov[2] = s->c22;
  cov[3] = s->c11;
  cov[4] = s->c31;
  cov[5] = s->c33;
}

/* velo_kalman_filter kernel (VeloKalmanFilter.cu:362-399) with linear_fit (:333-353) */
static void kalman_filter(
  unsigned n_events, const unsigned* offsets_all, const unsigned* offsets_hit_number, const char* track_hits,
  const float beamline[2], uint8_t* is_backward, float* beamline_states, float* endvelo_states)
{
  const unsigned total_tracks = offsets_all[n_events];
  const unsigned total_hits = offsets_hit_number[total_tracks];
  const float* coords = (const float*) track_hits + total_hits;
  for (unsigned i = 0; i < total_tracks; ++i) {
    KalmanTrack t = {coords + 3u * offsets_hit_number[i], offsets_hit_number[i + 1] - offsets_hit_number[i]};
    const float* first = t.xyz;
    const float* last = t.xyz + 3u * (t.n - 1);
    const float tx = (last[0] - first[0]) / (last[2] - first[2]);
    const float ty = (last[1] - first[1]) / (last[2] - first[2]);
    const float delta_z = (tx * (beamline[0] - last[0]) + ty * (beamline[1] - last[1])) / (tx * tx + ty * ty);
    const float lin_z = last[2] + delta_z;
    const int backward = lin_z > first[2];
    is_backward[i] = (uint8_t) backward;
    const KalmanState b = simplified_fit(&t, tx, ty, beamline, backward, 1);
    const KalmanState e = simplified_fit(&t, b.tx, b.ty, beamline, backward, 0);
    store_state(beamline_states, total_tracks, i, &b);
    store_state(endvelo_states, total_tracks, i, &e);
  }
}

void* velo_oracle_run(const VeloCpuInput* in)
{
  if (in->mep_layout) return NULL; /* the restatement reads the Allen layout only */
  Result* r = calloc(1, sizeof(Result));
  const unsigned n = in->n_events;
  Geometry* g = malloc(sizeof(Geometry));
  if (!parse_geometry(in->geometry, in->geometry_size, g)) memset(g, 0, sizeof(Geometry));
  uint8_t patterns[256];
  float sp_fx[512], sp_fy[512];
  sp_tables(patterns, sp_fx, sp_fy);

  unsigned total_clusters = 0;
  unsigned* offsets_est = NULL;
  unsigned* cluster_num = NULL;
  char* sorted = NULL;
  if (in->retina_decoding) {
    const unsigned per_event = retina_sensors_per_event(in->bank_version);
    unsigned* pair_size = make(r, "dev_each_sensor_pair_size", (size_t) n * per_event * sizeof(unsigned));
    unsigned* retina_bank_index = make(r, "dev_retina_bank_index", per_event * sizeof(unsigned));
    if (in->bank_version >= 0) retina_count(in, pair_size, retina_bank_index);
    unsigned* pair_offsets;
    total_clusters = prefix_sum(r, "dev_offsets_each_sensor_pair_size", pair_size, (size_t) n * per_event, &pair_offsets);
    cluster_num = make(r, "dev_module_cluster_num", (size_t) n * N_MODULE_PAIRS * sizeof(unsigned));
    offsets_est = make(r, "dev_offsets_estimated_input_size", ((size_t) n * N_MODULE_PAIRS + 1) * sizeof(unsigned));
    sorted = make(r, "dev_sorted_velo_cluster_container", (size_t) total_clusters * ELEMENT_SIZE);
    unsigned* permutations = make(r, "dev_hit_permutations", (size_t) total_clusters * sizeof(unsigned));
    int64_t* keys = make(r, "dev_hit_sorting_key", (size_t) total_clusters * sizeof(int64_t));
    if (in->bank_version >= 0)
      decode_retinaclusters(in, g, pair_offsets, retina_bank_index, cluster_num, offsets_est, sorted, permutations, keys);
  }
  else {
    unsigned* n_cand = make(r, "dev_number_of_candidates", n * sizeof(unsigned));
    unsigned* bank_index = make(r, "dev_velo_bank_index", N_SENSORS * sizeof(unsigned));
    if (in->bank_version >= 0) calculate_number_of_candidates(in, n_cand, bank_index);

    unsigned* cand_offsets;
    const unsigned total_cand = prefix_sum(r, "dev_candidates_offsets", n_cand, n, &cand_offsets);

    unsigned* estimated = make(r, "dev_estimated_input_size", (size_t) n * N_MODULE_PAIRS * sizeof(unsigned));
    unsigned* cand_num = make(r, "dev_module_candidate_num", n * sizeof(unsigned));
    uint32_t* candidates = make(r, "dev_cluster_candidates", (size_t) total_cand * sizeof(uint32_t));
    if (in->bank_version >= 0) estimate_input_size(in, cand_offsets, estimated, cand_num, candidates);

    total_clusters =
      prefix_sum(r, "dev_offsets_estimated_input_size", estimated, (size_t) n * N_MODULE_PAIRS, &offsets_est);

    cluster_num = make(r, "dev_module_cluster_num", (size_t) n * N_MODULE_PAIRS * sizeof(unsigned));
    char* container = make(r, "dev_velo_cluster_container", (size_t) total_clusters * ELEMENT_SIZE);
    if (in->bank_version >= 0)
      masked_clustering(
        in, g, patterns, sp_fx, sp_fy, offsets_est, cand_num, candidates, cand_offsets, bank_index, cluster_num,
        container);

    sorted = make(r, "dev_sorted_velo_cluster_container", (size_t) total_clusters * ELEMENT_SIZE);
    unsigned* perm = make(r, "dev_hit_permutation", (size_t) total_clusters * sizeof(unsigned));
    sort_by_phi(n, offsets_est, cluster_num, container, sorted, perm);
  }

  const unsigned by_clusters = (unsigned) ((float) total_clusters * tracks_per_cluster);
  const unsigned track_container_size =
    (float) total_clusters * tracks_per_cluster < (float) (n * MIN_CONTAINER) ? n * MIN_CONTAINER : by_clusters;
  TrackHits* tracks = make(r, "dev_tracks", (size_t) track_container_size * sizeof(TrackHits));
  TrackletHits* three_hit = make(r, "dev_three_hit_tracks", (size_t) track_container_size * sizeof(TrackletHits));
  TrackletHits* tracklets = make(r, "dev_tracklets", (size_t) n * MAX_TTF * sizeof(TrackletHits));
  unsigned* ttf = make(r, "dev_tracks_to_follow", (size_t) n * MAX_TTF * sizeof(unsigned));
  bool* hit_used = make(r, "dev_hit_used", (size_t) total_clusters);
  unsigned* atomics = make(r, "dev_atomics_velo", (size_t) n * 3 * sizeof(unsigned));
  unsigned* n_tracks = make(r, "dev_number_of_velo_tracks", n * sizeof(unsigned));
  uint16_t* rel = make(r, "dev_rel_indices", (size_t) total_clusters * sizeof(uint16_t));
  search_by_triplet(
    in, g, offsets_est, cluster_num, sorted, tracks, tracklets, ttf, three_hit, hit_used, atomics, rel, n_tracks);

  unsigned* offsets_tracks;
  const unsigned n_four = prefix_sum(r, "dev_offsets_velo_tracks", n_tracks, n, &offsets_tracks);

  TrackletHits* three_out =
    make(r, "dev_three_hit_tracks_output", (size_t) track_container_size * sizeof(TrackletHits));
  unsigned* n_three_out = make(r, "dev_number_of_three_hit_tracks_output", n * sizeof(unsigned));
  three_hit_tracks_filter(in, offsets_est, sorted, three_hit, atomics, hit_used, three_out, n_three_out);

  unsigned* offsets_three;
  const unsigned n_three =
    prefix_sum(r, "dev_offsets_number_of_three_hit_tracks_filtered", n_three_out, n, &offsets_three);

  unsigned* hit_number = make(r, "dev_velo_track_hit_number", (size_t) (n_four + n_three) * sizeof(unsigned));
  unsigned* offsets_all = make(r, "dev_offsets_all_velo_tracks", (n + 1) * sizeof(unsigned));
  copy_track_hit_number(n, offsets_est, tracks, offsets_tracks, offsets_three, hit_number, offsets_all);
  unsigned* host_reco = make(r, "host_number_of_reconstructed_velo_tracks", sizeof(unsigned));
  *host_reco = offsets_all[n];

  unsigned* offsets_hit_number;
  const unsigned total_track_hits =
    prefix_sum(r, "dev_offsets_velo_track_hit_number", hit_number, n_four + n_three, &offsets_hit_number);

  /* sized as VeloConsolidateTracks.cu:53-58 does: reconstructed tracks (which already
   * include the three-hit ones) plus the three-hit tracks once more */
  const unsigned total_tracks = offsets_all[n] + n_three;
  uint8_t* accepted = make(r, "dev_accepted_velo_tracks", total_tracks);
  memset(accepted, 1, total_tracks);
  char* track_hits = make(r, "dev_velo_track_hits", (size_t) total_track_hits * ELEMENT_SIZE);
  consolidate_tracks(
    n, offsets_est, offsets_all, tracks, offsets_hit_number, sorted, three_out, offsets_three, track_hits);

  /* velo_kalman_filter (VeloKalmanFilter.cu:8-18 sizes) */
  const unsigned reco = offsets_all[n];
  const float beamline[2] = {in->beamline_x, in->beamline_y};
  uint8_t* is_backward = make(r, "dev_is_backward", reco);
  float* beamline_states = make(r, "dev_velo_kalman_beamline_states", (size_t) reco * 56u);
  float* endvelo_states = make(r, "dev_velo_kalman_endvelo_states", (size_t) reco * 56u);
  kalman_filter(n, offsets_all, offsets_hit_number, track_hits, beamline, is_backward, beamline_states, endvelo_states);
  free(g);
  return r;
}

const void* velo_oracle_get(void* handle, const char* name, size_t* nbytes)
{
  Result* r = handle;
  for (int i = 0; i < r->count; ++i) {
    if (!strcmp(r->b[i].name, name)) {
      if (nbytes) *nbytes = r->b[i].n;
      return r->b[i].p;
    }
  }
  if (nbytes) *nbytes = 0;
  return NULL;
}

void velo_oracle_free(void* handle)
{
  Result* r = handle;
  if (!r) return;
  for (int i = 0; i < r->count; ++i)
    free(r->b[i].p);
  free(r);
}

typedef struct {
  const VeloCpuInput* in;
  unsigned slice_size, n_slices, n_threads, thread;
} TimeArgs;

static void* time_worker(void* arg)
{
  const TimeArgs* a = arg;
  /* slices cycle over the events available, so a sample may be longer than the input */
  const unsigned available = a->in->n_events / a->slice_size ? a->in->n_events / a->slice_size : 1;
  for (unsigned s = a->thread; s < a->n_slices; s += a->n_threads) {
    VeloCpuInput slice = *a->in;
    slice.event_start = a->in->event_start + (s % available) * a->slice_size;
    slice.n_events = a->slice_size;
    velo_oracle_free(velo_oracle_run(&slice));
  }
  return NULL;
}

/* Wall seconds for n_slices slices of slice_size events over n_threads threads. */
double velo_oracle_time(const VeloCpuInput* in, unsigned slice_size, unsigned n_slices, unsigned n_threads)
{
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  pthread_t th[256];
  TimeArgs args[256];
  if (n_threads > 256) n_threads = 256;
  for (unsigned t = 0; t < n_threads; ++t) {
    args[t] = (TimeArgs) {in, slice_size, n_slices, n_threads, t};
    pthread_create(&th[t], NULL, time_worker, &args[t]);
  }
  for (unsigned t = 0; t < n_threads; ++t)
    pthread_join(th[t], NULL);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  return (double) (t1.tv_sec - t0.tv_sec) + 1e-9 * (double) (t1.tv_nsec - t0.tv_nsec);
}
