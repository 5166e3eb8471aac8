// The crate's on-disk SDF format, version V1 (serde.rs:106-221), host side.
//
// save_to_file writes `rmp_serde::to_vec(&SerializeVersion::V1(sdf))`: with
// rmp-serde's default configuration an enum is a one-entry map from the
// variant name to its value and a struct is an array of its fields, so
//   Generic: {"V1": {"Generic": [query_points, distances]}}
//   Grid:    {"V1": {"Grid": [[first_cell, cell_size, cell_count], distances]}}
// with a point as an array of three f32, every f32 as msgpack float 32
// (0xca), cell counts (usize) as the shortest msgpack unsigned integer, and
// every length in its shortest form (the msgpack specification).  The reader
// accepts what rmp-serde's reader accepts for these types as well: floats of
// 64 bits and integers where an f32 is expected, any integer width for counts,
// and structs written as maps of field names.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "m2s_internal.cuh"

using namespace m2s;

namespace {

struct Writer {
  uint8_t* out;  // NULL: only count
  uint64_t cap, len = 0;
  void byte(uint8_t b) {
    if (out && len < cap) out[len] = b;
    ++len;
  }
  void be(uint64_t v, int bytes) {
    for (int i = bytes - 1; i >= 0; --i) byte((uint8_t)(v >> (8 * i)));
  }
  void map(uint32_t n) {
    if (n < 16) byte(0x80 | n);
    else if (n < 65536) byte(0xde), be(n, 2);
    else byte(0xdf), be(n, 4);
  }
  void array(uint64_t n) {
    if (n < 16) byte(0x90 | (uint8_t)n);
    else if (n < 65536) byte(0xdc), be(n, 2);
    else byte(0xdd), be(n, 4);
  }
  void str(const char* s) {
    const size_t n = strlen(s);
    if (n < 32) byte(0xa0 | (uint8_t)n);
    else if (n < 256) byte(0xd9), be(n, 1);
    else byte(0xda), be(n, 2);
    for (size_t i = 0; i < n; ++i) byte((uint8_t)s[i]);
  }
  void f32(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    byte(0xca);
    be(b, 4);
  }
  void uint(uint64_t u) {
    if (u < 128) byte((uint8_t)u);
    else if (u < 256) byte(0xcc), be(u, 1);
    else if (u < 65536) byte(0xcd), be(u, 2);
    else if (u < (1ull << 32)) byte(0xce), be(u, 4);
    else byte(0xcf), be(u, 8);
  }
  void point(const float* p) {
    array(3);
    for (int d = 0; d < 3; ++d) f32(p[d]);
  }
  void floats(const float* v, uint64_t n) {
    array(n);
    for (uint64_t i = 0; i < n; ++i) f32(v[i]);
  }
};

int finish(const Writer& w, uint8_t* out, uint64_t capacity, uint64_t* out_len) {
  *out_len = w.len;
  if (out && w.len > capacity) {
    set_error("serialize: the output buffer holds " + std::to_string(capacity) + " bytes, " +
              std::to_string(w.len) + " are needed");
    return M2S_ERR_INVALID_ARGUMENT;
  }
  return M2S_OK;
}

// ---- reader -------------------------------------------------------------------
struct Reader {
  const uint8_t* p;
  uint64_t n, pos = 0;
  bool ok = true;
  bool need(uint64_t k) {
    if (!ok || pos + k > n) ok = false;
    return ok;
  }
  uint64_t be(int bytes) {
    if (!need(bytes)) return 0;
    uint64_t v = 0;
    for (int i = 0; i < bytes; ++i) v = (v << 8) | p[pos++];
    return v;
  }
  uint8_t peek() { return need(1) ? p[pos] : 0; }
  // Header of a map or array; returns false on another type.
  bool map(uint64_t* len) {
    const uint8_t b = peek();
    if (!ok) return false;
    if ((b & 0xf0) == 0x80) return ++pos, *len = b & 0x0f, true;
    if (b == 0xde) return ++pos, *len = be(2), ok;
    if (b == 0xdf) return ++pos, *len = be(4), ok;
    return false;
  }
  bool array(uint64_t* len) {
    const uint8_t b = peek();
    if (!ok) return false;
    if ((b & 0xf0) == 0x90) return ++pos, *len = b & 0x0f, true;
    if (b == 0xdc) return ++pos, *len = be(2), ok;
    if (b == 0xdd) return ++pos, *len = be(4), ok;
    return false;
  }
  bool str(std::string* s) {
    const uint8_t b = peek();
    if (!ok) return false;
    uint64_t len;
    if ((b & 0xe0) == 0xa0) ++pos, len = b & 0x1f;
    else if (b == 0xd9) ++pos, len = be(1);
    else if (b == 0xda) ++pos, len = be(2);
    else if (b == 0xdb) ++pos, len = be(4);
    else return false;
    if (!need(len)) return false;
    s->assign((const char*)p + pos, len);
    pos += len;
    return true;
  }
  // A number as f32 (float 32/64 or an integer, as serde's f32 visitor takes them).
  bool f32(float* f) {
    const uint8_t b = peek();
    if (!ok) return false;
    if (b == 0xca) {
      ++pos;
      const uint32_t v = (uint32_t)be(4);
      memcpy(f, &v, 4);
      return ok;
    }
    if (b == 0xcb) {
      ++pos;
      const uint64_t v = be(8);
      double d;
      memcpy(&d, &v, 8);
      *f = (float)d;
      return ok;
    }
    int64_t i;
    if (!integer(&i)) return false;
    *f = (float)i;
    return true;
  }
  bool integer(int64_t* v) {
    const uint8_t b = peek();
    if (!ok) return false;
    if (b < 0x80) return ++pos, *v = b, true;
    if (b >= 0xe0) return ++pos, *v = (int8_t)b, true;
    switch (b) {
      case 0xcc: ++pos; *v = (int64_t)be(1); return ok;
      case 0xcd: ++pos; *v = (int64_t)be(2); return ok;
      case 0xce: ++pos; *v = (int64_t)be(4); return ok;
      case 0xcf: ++pos; *v = (int64_t)be(8); return ok;  // values above i64 are refused below
      case 0xd0: ++pos; *v = (int8_t)be(1); return ok;
      case 0xd1: ++pos; *v = (int16_t)be(2); return ok;
      case 0xd2: ++pos; *v = (int32_t)be(4); return ok;
      case 0xd3: ++pos; *v = (int64_t)be(8); return ok;
      default: return false;
    }
  }
  bool usize(uint64_t* u) {
    const uint8_t b = peek();
    if (b == 0xcf) {
      ++pos;
      *u = be(8);
      return ok;
    }
    int64_t v;
    if (!integer(&v) || v < 0) return false;
    *u = (uint64_t)v;
    return true;
  }
  bool point(float* out3) {
    uint64_t len;
    if (array(&len)) {
      if (len != 3) return false;
      for (int d = 0; d < 3; ++d)
        if (!f32(out3 + d)) return false;
      return true;
    }
    if (map(&len)) {  // a struct written with field names: {"x": .., "y": .., "z": ..}
      if (len != 3) return false;
      for (uint64_t k = 0; k < 3; ++k) {
        std::string key;
        if (!str(&key) || key.size() != 1 || key[0] < 'x' || key[0] > 'z') return false;
        if (!f32(out3 + (key[0] - 'x'))) return false;
      }
      return true;
    }
    return false;
  }
};

struct Parsed {
  int kind = -1;  // 0 generic, 1 grid
  std::vector<float> points, distances;
  float first[3] = {0, 0, 0}, size[3] = {0, 0, 0};
  uint64_t count[3] = {0, 0, 0};
};

bool read_floats(Reader& r, std::vector<float>* out) {
  uint64_t n;
  if (!r.array(&n) || n > r.n) return false;  // every element takes at least one byte
  out->resize(n);
  for (uint64_t i = 0; i < n; ++i)
    if (!r.f32(&(*out)[i])) return false;
  return true;
}

bool read_points(Reader& r, std::vector<float>* out) {
  uint64_t n;
  if (!r.array(&n) || n > r.n) return false;
  out->resize(3 * n);
  for (uint64_t i = 0; i < n; ++i)
    if (!r.point(&(*out)[3 * i])) return false;
  return true;
}

bool read_grid(Reader& r, Parsed* P) {
  uint64_t len;
  auto counts = [&]() {
    uint64_t m;
    if (!r.array(&m) || m != 3) return false;
    for (int d = 0; d < 3; ++d)
      if (!r.usize(&P->count[d])) return false;
    return true;
  };
  if (r.array(&len)) {
    return len == 3 && r.point(P->first) && r.point(P->size) && counts();
  }
  if (!r.map(&len) || len != 3) return false;
  bool seen[3] = {false, false, false};
  for (uint64_t k = 0; k < 3; ++k) {
    std::string key;
    if (!r.str(&key)) return false;
    if (key == "first_cell" && !seen[0]) seen[0] = r.point(P->first);
    else if (key == "cell_size" && !seen[1]) seen[1] = r.point(P->size);
    else if (key == "cell_count" && !seen[2]) seen[2] = counts();
    else return false;
  }
  return seen[0] && seen[1] && seen[2];
}

// [field0, field1] or {"name0": field0, "name1": field1}
template <class F0, class F1>
bool read_pair(Reader& r, const char* name0, const char* name1, F0 f0, F1 f1) {
  uint64_t len;
  if (r.array(&len)) return len == 2 && f0() && f1();
  if (!r.map(&len) || len != 2) return false;
  bool a = false, b = false;
  for (int k = 0; k < 2; ++k) {
    std::string key;
    if (!r.str(&key)) return false;
    if (key == name0 && !a) a = f0();
    else if (key == name1 && !b) b = f1();
    else return false;
  }
  return a && b;
}

bool parse(const uint8_t* data, uint64_t n, Parsed* P) {
  Reader r{data, n};
  uint64_t len;
  std::string key;
  if (!r.map(&len) || len != 1 || !r.str(&key) || key != "V1") return false;
  if (!r.map(&len) || len != 1 || !r.str(&key)) return false;
  bool ok;
  if (key == "Generic") {
    P->kind = 0;
    ok = read_pair(
        r, "query_points", "distances", [&] { return read_points(r, &P->points); },
        [&] { return read_floats(r, &P->distances); });
  } else if (key == "Grid") {
    P->kind = 1;
    ok = read_pair(
        r, "grid", "distances", [&] { return read_grid(r, P); }, [&] { return read_floats(r, &P->distances); });
  } else {
    return false;
  }
  return ok && r.ok && r.pos == n;
}

}  // namespace

extern "C" {

int m2s_serialize_generic(const float* query_points, uint64_t n_points, const float* distances, uint64_t n_distances,
                          uint8_t* out, uint64_t capacity, uint64_t* out_len) {
  if (!out_len || (n_points && !query_points) || (n_distances && !distances)) return M2S_ERR_INVALID_ARGUMENT;
  if (n_points > 0xFFFFFFFFull || n_distances > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  Writer w{out, capacity};
  w.map(1);
  w.str("V1");
  w.map(1);
  w.str("Generic");
  w.array(2);
  w.array(n_points);
  for (uint64_t i = 0; i < n_points; ++i) w.point(query_points + 3 * i);
  w.floats(distances, n_distances);
  return finish(w, out, capacity, out_len);
}

int m2s_serialize_grid(const float first_cell[3], const float cell_size[3], const uint64_t cell_count[3],
                       const float* distances, uint64_t n_distances, uint8_t* out, uint64_t capacity,
                       uint64_t* out_len) {
  if (!out_len || !first_cell || !cell_size || !cell_count || (n_distances && !distances))
    return M2S_ERR_INVALID_ARGUMENT;
  if (n_distances > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  Writer w{out, capacity};
  w.map(1);
  w.str("V1");
  w.map(1);
  w.str("Grid");
  w.array(2);
  w.array(3);
  w.point(first_cell);
  w.point(cell_size);
  w.array(3);
  for (int d = 0; d < 3; ++d) w.uint(cell_count[d]);
  w.floats(distances, n_distances);
  return finish(w, out, capacity, out_len);
}

int m2s_deserialize(const uint8_t* data, uint64_t len, int* kind, uint64_t* n_points, uint64_t* n_distances,
                    float* query_points, float* distances, float grid_first[3], float grid_size[3],
                    uint64_t grid_count[3]) {
  if ((len && !data) || !kind || !n_points || !n_distances) return M2S_ERR_INVALID_ARGUMENT;
  Parsed P;
  if (!parse(data, len, &P)) {
    set_error("deserialize: not a V1 signed distance field");
    *kind = -1;
    return M2S_ERR_FORMAT;
  }
  *kind = P.kind;
  *n_points = P.points.size() / 3;
  *n_distances = P.distances.size();
  if (query_points && !P.points.empty()) memcpy(query_points, P.points.data(), 4 * P.points.size());
  if (distances && !P.distances.empty()) memcpy(distances, P.distances.data(), 4 * P.distances.size());
  if (P.kind == 1) {
    if (grid_first) memcpy(grid_first, P.first, 12);
    if (grid_size) memcpy(grid_size, P.size, 12);
    if (grid_count) memcpy(grid_count, P.count, 24);
  }
  return M2S_OK;
}

}  // extern "C"
