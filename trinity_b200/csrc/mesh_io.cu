/*
 * mesh_io.cu — host-side readers and writers of the mesh files
 * (Mesh::load, io.cpp:53-161; the .bb solution, io.cpp:106-135).
 *
 * The medit text format holds one record per line in practice (Vertices:
 * x y ref; Edges: a b ref; Triangles: a b c ref; Corners: v; the .bb values
 * one per line). The reader splits each section's byte range into newline-
 * aligned chunks, one per host thread: each thread counts the records of its
 * chunk, a prefix sum places them, and each thread then converts its own
 * lines with std::from_chars (correctly rounded, so the values are those of
 * strtod). A section that is not laid out one record per line (a record
 * split over lines, a stray token) makes the caller fall back to the
 * token-by-token reader.
 *
 * The binary form ("TRNB" files, trn_mesh_store_binary) stores the arrays
 * themselves: a 64-byte header, then the points (2 f64 a vertex), the
 * vertex tags (u8), the triangles (3 i32, 0-based). trn_mesh_load reads it
 * when a file starts with the magic, in place of the text form.
 */
#include "trn_internal.h"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace trn {

namespace {

inline bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

/* the numbers of one line [p, e): nd doubles then integers, nf in all;
 * false unless the line holds exactly nf numbers */
bool parse_line(const char* p, const char* e, int nf, int nd, double* dv, long* iv) {
  int k = 0;
  while (true) {
    while (p < e && is_blank(*p)) ++p;
    if (p >= e) break;
    if (k >= nf) return false;
    std::from_chars_result r;
    if (k < nd) r = std::from_chars(p, e, dv[k]);
    else r = std::from_chars(p, e, iv[k - nd]);
    if (r.ec != std::errc() || (r.ptr < e && !is_blank(*r.ptr))) return false;
    p = r.ptr;
    ++k;
  }
  return k == nf;
}

bool blank_line(const char* p, const char* e) {
  while (p < e && is_blank(*p)) ++p;
  return p >= e;
}

int host_threads() {
  const unsigned h = std::thread::hardware_concurrency();
  return (int) std::max(1u, std::min(h ? h : 1u, 32u));
}

}  // namespace

/* count records of nf numbers (one per non-blank line) starting at byte s;
 * on success *end is the byte after the last one. Records are handed to
 * put(k, dv, iv) with k = 0..count-1, in parallel. */
template <class Put>
static bool parse_section(const std::vector<char>& buf, size_t s, long count, int nf, int nd, Put put,
                          size_t* end) {
  const char* b = buf.data();
  const size_t n = buf.size() - 1;   /* the buffer ends with a 0 */
  /* the section's end: after `count` non-blank lines */
  size_t pos = s;
  long seen = 0;
  while (seen < count && pos < n) {
    const char* nl = static_cast<const char*>(std::memchr(b + pos, '\n', n - pos));
    const size_t eol = nl ? (size_t) (nl - b) : n;
    if (!blank_line(b + pos, b + eol)) ++seen;
    pos = eol < n ? eol + 1 : n;
  }
  if (seen < count) return false;
  *end = pos;
  const size_t len = pos - s;
  const int nt = (int) std::max<size_t>(1, std::min<size_t>((size_t) host_threads(), len >> 20));
  std::vector<size_t> cut((size_t) nt + 1);
  cut[0] = s;
  cut[(size_t) nt] = pos;
  for (int t = 1; t < nt; ++t) {
    size_t c = s + len * (size_t) t / (size_t) nt;
    const char* nl = static_cast<const char*>(std::memchr(b + c, '\n', pos - c));
    cut[(size_t) t] = nl ? (size_t) (nl - b) + 1 : pos;
  }
  std::vector<long> cnt((size_t) nt, 0);
  std::vector<char> ok((size_t) nt, 1);
  auto lines = [&](int t, auto fn) {
    size_t p = cut[(size_t) t];
    const size_t e = cut[(size_t) t + 1];
    while (p < e) {
      const char* nl = static_cast<const char*>(std::memchr(b + p, '\n', e - p));
      const size_t eol = nl ? (size_t) (nl - b) : e;
      if (!blank_line(b + p, b + eol) && !fn(b + p, b + eol)) return false;
      p = eol + 1;
    }
    return true;
  };
  auto run = [&](auto body) {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(body, t);
    body(0);
    for (auto& x : th) x.join();
  };
  run([&](int t) {
    long c = 0;
    lines(t, [&](const char*, const char*) { ++c; return true; });
    cnt[(size_t) t] = c;
  });
  std::vector<long> base((size_t) nt + 1, 0);
  for (int t = 0; t < nt; ++t) base[(size_t) t + 1] = base[(size_t) t] + cnt[(size_t) t];
  if (base[(size_t) nt] != count) return false;
  run([&](int t) {
    long k = base[(size_t) t];
    ok[(size_t) t] = lines(t, [&](const char* p, const char* e) {
      double dv[4];
      long iv[4];
      if (!parse_line(p, e, nf, nd, dv, iv)) return false;
      put(k++, dv, iv);
      return true;
    }) ? 1 : 0;
  });
  for (char x : ok)
    if (!x) return false;
  return true;
}

/* the first line at or after *pos whose first token is key (io::find,
 * io.cpp:25-49); *pos moves past it and the count is parsed from the rest
 * of the buffer; -1 when absent */
static long find_section(const std::vector<char>& buf, size_t* pos, const char* key) {
  const char* b = buf.data();
  const size_t n = buf.size() - 1, klen = std::strlen(key);
  size_t p = *pos;
  while (p < n) {
    const char* nl = static_cast<const char*>(std::memchr(b + p, '\n', n - p));
    const size_t eol = nl ? (size_t) (nl - b) : n;
    size_t q = p;
    while (q < eol && is_blank(b[q])) ++q;
    const bool hit = q < eol && b[q] != '#' && b[q] != '%' && eol - q >= klen &&
                     std::strncmp(b + q, key, klen) == 0 && (q + klen == eol || is_blank(b[q + klen]));
    p = eol < n ? eol + 1 : n;
    if (hit) {
      /* the count: the next token, possibly on the following line */
      while (p < n && (is_blank(b[p]) || b[p] == '\n')) ++p;
      long c = -1;
      auto r = std::from_chars(b + p, b + n, c);
      if (r.ec != std::errc()) return -1;
      p = (size_t) (r.ptr - b);
      while (p < n && b[p] != '\n') ++p;
      *pos = p < n ? p + 1 : n;
      return c;
    }
  }
  *pos = n;
  return -1;
}

bool read_file(const char* path, std::vector<char>* buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  buf->resize((size_t) (n > 0 ? n : 0) + 1);
  const size_t got = n > 0 ? std::fread(buf->data(), 1, (size_t) n, f) : 0;
  std::fclose(f);
  (*buf)[got] = 0;
  buf->resize(got + 1);
  return true;
}

static constexpr char kBinMagic[8] = {'T', 'R', 'N', 'B', '0', '0', '0', '1'};

int parse_mesh_text(const std::vector<char>& buf, MeshInput* out, std::string* err) {
  size_t pos = 0;
  const long nv = find_section(buf, &pos, "Vertices");
  if (nv <= 0) { *err = "mesh: no Vertices section"; return 1; }
  out->pts.assign((size_t) nv * 2, 0.0);
  out->tags.assign((size_t) nv, 0);
  size_t end = 0;
  if (!parse_section(buf, pos, nv, 3, 2, [&](long k, const double* dv, const long*) {
        out->pts[2 * (size_t) k] = dv[0];
        out->pts[2 * (size_t) k + 1] = dv[1];
      }, &end))
    return -1;
  const size_t after_v = end;
  pos = after_v;
  const long ne = find_section(buf, &pos, "Edges");
  std::vector<long> bnd;
  if (ne > 0) {
    bnd.assign((size_t) ne * 2, 0);
    if (!parse_section(buf, pos, ne, 3, 0, [&](long k, const double*, const long* iv) {
          bnd[2 * (size_t) k] = iv[0];
          bnd[2 * (size_t) k + 1] = iv[1];
        }, &end))
      return -1;
    for (long v : bnd)
      if (v < 1 || v > nv) { *err = "mesh: edge index out of range"; return 1; }
    for (long v : bnd) out->tags[(size_t) v - 1] = TRN_TAG_BOUND;
    pos = end;
  } else {
    pos = after_v;
  }
  const long nt = find_section(buf, &pos, "Triangles");
  if (nt <= 0) { *err = "mesh: no Triangles section"; return 1; }
  out->tris.assign((size_t) nt * 3, 0);
  if (!parse_section(buf, pos, nt, 4, 0, [&](long k, const double*, const long* iv) {
        out->tris[3 * (size_t) k] = (int) iv[0] - 1;
        out->tris[3 * (size_t) k + 1] = (int) iv[1] - 1;
        out->tris[3 * (size_t) k + 2] = (int) iv[2] - 1;
      }, &end))
    return -1;
  const size_t after_t = end;
  pos = after_t;
  const long nc = find_section(buf, &pos, "Corners");
  if (nc > 0) {
    std::vector<long> cor((size_t) nc);
    if (!parse_section(buf, pos, nc, 1, 0, [&](long k, const double*, const long* iv) { cor[(size_t) k] = iv[0]; },
                       &end))
      return -1;
    for (long v : cor)
      if (v < 1 || v > nv) { *err = "mesh: corner index out of range"; return 1; }
    for (long v : cor) out->tags[(size_t) v - 1] = TRN_TAG_BOUND | TRN_TAG_CORNER;
  }
  out->nv = nv;
  out->nt = nt;
  return 0;
}

int parse_bb_text(const std::vector<char>& buf, long nv, std::vector<double>* u, std::string* err) {
  /* header "dim nb_sol nb_values type" (io.cpp:114-118) on the first line */
  const char* b = buf.data();
  const size_t n = buf.size() - 1;
  size_t p = 0;
  long hdr[4];
  for (int k = 0; k < 4; ++k) {
    while (p < n && (is_blank(b[p]) || b[p] == '\n')) ++p;
    auto r = std::from_chars(b + p, b + n, hdr[k]);
    if (r.ec != std::errc()) { *err = "bb: bad header"; return 1; }
    p = (size_t) (r.ptr - b);
  }
  if (hdr[2] != nv) { *err = "bb: wrong number of vertices in solution file"; return 1; }
  while (p < n && b[p] != '\n') ++p;
  if (p < n) ++p;
  u->assign((size_t) nv, 0.0);
  size_t end = 0;
  if (!parse_section(buf, p, nv, 1, 1, [&](long k, const double* dv, const long*) { (*u)[(size_t) k] = dv[0]; },
                     &end))
    return -1;
  return 0;
}

bool is_binary_mesh(const std::vector<char>& buf) {
  return buf.size() > 64 && std::memcmp(buf.data(), kBinMagic, 8) == 0;
}

int parse_mesh_binary(const std::vector<char>& buf, MeshInput* out, std::string* err) {
  long long hdr[8];
  std::memcpy(hdr, buf.data(), sizeof(hdr));
  const long long nv = hdr[1], nt = hdr[2];
  const size_t need = 64 + (size_t) nv * 17 + (size_t) nt * 12;
  if (nv <= 0 || nt <= 0 || buf.size() - 1 < need) { *err = "binary mesh: truncated"; return 1; }
  const char* p = buf.data() + 64;
  out->pts.resize((size_t) nv * 2);
  std::memcpy(out->pts.data(), p, (size_t) nv * 16);
  p += (size_t) nv * 16;
  out->tags.resize((size_t) nv);
  std::memcpy(out->tags.data(), p, (size_t) nv);
  p += (size_t) nv;
  out->tris.resize((size_t) nt * 3);
  std::memcpy(out->tris.data(), p, (size_t) nt * 12);
  out->nv = (long) nv;
  out->nt = (long) nt;
  return 0;
}

int write_mesh_binary(const char* path, long nv, long nt, const double* pts, const uint8_t* tags,
                      const int* tris) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return 1;
  long long hdr[8] = {0, nv, nt, 0, 0, 0, 0, 0};
  std::memcpy(hdr, kBinMagic, 8);
  bool ok = std::fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
            std::fwrite(pts, 16, (size_t) nv, f) == (size_t) nv &&
            std::fwrite(tags, 1, (size_t) nv, f) == (size_t) nv &&
            std::fwrite(tris, 12, (size_t) nt, f) == (size_t) nt;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : 1;
}

}  // namespace trn
