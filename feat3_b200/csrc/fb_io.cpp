// Container file I/O in FEAT3's own formats (host code of the C-ABI library).
//
// Hierarchies, right-hand sides and solutions move between a FEAT3 application and this
// library as files in the formats the reference writes and reads:
//   * fm_csr / fm_binary : the serialised container (Container::_serialise / _deserialise,
//     kernel/lafem/container.hpp:317-572) of SparseMatrixCSR, stored as double values and
//     uint64 indices whatever the in-memory types (sparse_matrix_csr.hpp:1243-1245, 1267-1269);
//   * fm_dv / fm_binary  : the serialised DenseVector (dense_vector.hpp:706-708, 772-774);
//   * fm_mtx             : MatrixMarket text, "coordinate real general|symmetric" for matrices
//     (sparse_matrix_csr.hpp:1120-1241, 1296-1339), "array real general" for vectors
//     (dense_vector.hpp:609-667, 744-759);
//   * fm_exp             : one value per line, lines holding '#' skipped (dense_vector.hpp:
//     669-705, 760-771);
//   * fm_mtx sparse vectors ("coordinate real general", one column): a UnitFilter's Dirichlet list
//     (sparse_vector.hpp:517-680).
// The byte layout has to be the reference's so that files cross between the two programs; the
// parsing and formatting code is this library's own (a counting-sort CSR build instead of the
// reference's ordered map, std::to_chars for the "%.6e" text of std::scientific).
//
// Where the reference leaves an input undefined this code rejects it with FB_ERR_FORMAT
// instead: entry indices outside the declared dimensions, duplicate entries (the reference
// keeps the first but counts both, leaving row_ptr inconsistent), a vector file holding more
// or fewer values than its header, serialised arrays that do not fit the stated size. Beyond
// the reference it builds correct row pointers for rows without entries, accepts tabs and
// carriage returns as separators, skips blank lines before the size line and parses a last
// line that has no line feed.
#include "feat3_b200.h"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

// LAFEM::FileMode values (kernel/lafem/base.hpp:31-46); the serialised magic number is the
// enum value of fm_csr resp. fm_dv.
constexpr uint64_t kMagicCsr = FB_FILE_CSR;
constexpr uint64_t kMagicDv = FB_FILE_DV;
// Type::Traits<T>::feature_hash (kernel/util/type_traits.hpp:121-124, 155-158, 427-430):
// sizeof | is_int << 32 | is_float << 33 | is_signed << 34 of double and Index (unsigned long).
constexpr uint64_t kIntBit = uint64_t(1) << 32, kFloatBit = uint64_t(1) << 33, kSignBit = uint64_t(1) << 34;
constexpr uint64_t kHashDouble = 8 | kFloatBit | kSignBit;
constexpr uint64_t kHashIndex = 8 | kIntBit;
constexpr uint64_t kHeaderWords = 10;  // size, magic, two hashes, six array counts
constexpr uint64_t kPadBytes = 16;     // trailing padding of the serialised array

// ---------------------------------------------------------------------------------------------
// serialised container: layout of Container::_serialise for 8-byte value and index types
struct Parts {
  std::vector<uint64_t> elements_size, indices_size, scalar_index;
  std::vector<double> scalar_dt;
  std::vector<const void*> elements, indices;  // arrays of elements_size[i] doubles / indices_size[i] u64
};

uint64_t serialised_size(const Parts& p)
{
  uint64_t words = kHeaderWords + p.elements_size.size() + p.indices_size.size() + p.scalar_index.size() +
                   p.scalar_dt.size();
  for(uint64_t s : p.elements_size) words += s;
  for(uint64_t s : p.indices_size) words += s;
  return words * 8 + kPadBytes;
}

// byte sink: a caller buffer or a FILE*
struct Sink {
  char* buf = nullptr;
  uint64_t pos = 0, cap = 0;
  FILE* f = nullptr;
  bool ok = true;
  void put(const void* p, uint64_t bytes)
  {
    if(!ok || bytes == 0) return;
    if(f) { ok = std::fwrite(p, 1, bytes, f) == bytes; return; }
    if(pos + bytes > cap) { ok = false; return; }
    std::memcpy(buf + pos, p, bytes);
    pos += bytes;
  }
  void put_u64(uint64_t v) { put(&v, 8); }
};

void serialise(Sink& s, const Parts& p, uint64_t magic)
{
  s.put_u64(serialised_size(p));
  s.put_u64(magic);
  s.put_u64(kHashDouble);
  s.put_u64(kHashIndex);
  s.put_u64(p.elements.size());
  s.put_u64(p.indices.size());
  s.put_u64(p.elements_size.size());
  s.put_u64(p.indices_size.size());
  s.put_u64(p.scalar_index.size());
  s.put_u64(p.scalar_dt.size());
  for(uint64_t v : p.elements_size) s.put_u64(v);
  for(uint64_t v : p.indices_size) s.put_u64(v);
  for(uint64_t v : p.scalar_index) s.put_u64(v);
  for(double v : p.scalar_dt) s.put(&v, 8);
  for(size_t i = 0; i < p.elements.size(); ++i) s.put(p.elements[i], p.elements_size[i] * 8);
  for(size_t i = 0; i < p.indices.size(); ++i) s.put(p.indices[i], p.indices_size[i] * 8);
  static const char zeros[kPadBytes] = {};
  s.put(zeros, kPadBytes);
}

// Parse a serialised container held in buf[0, avail). On success the views point into buf.
int deserialise(const char* buf, uint64_t avail, uint64_t magic, Parts& p)
{
  if(avail < kHeaderWords * 8) return FB_ERR_FORMAT;
  uint64_t h[kHeaderWords];
  std::memcpy(h, buf, sizeof(h));
  const uint64_t gsize = h[0];
  if(gsize > avail || gsize < kHeaderWords * 8 || gsize % 8 != 0) return FB_ERR_FORMAT;
  if(h[1] != magic) return FB_ERR_FORMAT;
  // the value type must be a signed floating type, the index type an unsigned integer type
  // (the reference asserts these features and only warns about differing sizes)
  if((h[2] & (kIntBit | kFloatBit | kSignBit)) != (kFloatBit | kSignBit)) return FB_ERR_FORMAT;
  if((h[3] & (kIntBit | kFloatBit | kSignBit)) != kIntBit) return FB_ERR_FORMAT;
  if(h[4] != h[6] || h[5] != h[7]) return FB_ERR_FORMAT;
  const uint64_t words = gsize / 8;
  uint64_t w = kHeaderWords;
  const uint64_t counts = h[6] + h[7] + h[8] + h[9];
  if(h[6] > words || h[7] > words || h[8] > words || h[9] > words || w + counts > words) return FB_ERR_FORMAT;
  auto word = [&](uint64_t i) { uint64_t v; std::memcpy(&v, buf + 8 * i, 8); return v; };
  p = Parts();
  for(uint64_t i = 0; i < h[6]; ++i) p.elements_size.push_back(word(w++));
  for(uint64_t i = 0; i < h[7]; ++i) p.indices_size.push_back(word(w++));
  for(uint64_t i = 0; i < h[8]; ++i) p.scalar_index.push_back(word(w++));
  for(uint64_t i = 0; i < h[9]; ++i) { double d; std::memcpy(&d, buf + 8 * w++, 8); p.scalar_dt.push_back(d); }
  for(uint64_t s : p.elements_size) {
    if(s > words - w) return FB_ERR_FORMAT;
    p.elements.push_back(buf + 8 * w);
    w += s;
  }
  for(uint64_t s : p.indices_size) {
    if(s > words - w) return FB_ERR_FORMAT;
    p.indices.push_back(buf + 8 * w);
    w += s;
  }
  return FB_OK;
}

template <typename T>
T* alloc_copy(const void* src, uint64_t n)
{
  T* dst = static_cast<T*>(std::malloc(std::max<uint64_t>(n, 1) * sizeof(T)));
  if(dst && n) std::memcpy(dst, src, n * sizeof(T));
  return dst;
}

void csr_free(fb_csr_host* m)
{
  std::free(const_cast<uint64_t*>(m->row_ptr));
  std::free(const_cast<uint64_t*>(m->col_ind));
  std::free(const_cast<double*>(m->val));
  *m = fb_csr_host{};
}

// checks a caller CSR (row pointers monotone from 0 to nnz, columns in range)
int csr_check(const fb_csr_host* m)
{
  if(!m) return FB_ERR_INVALID;
  if(m->rows == 0) return m->nnz == 0 ? FB_OK : FB_ERR_INVALID;
  if(!m->row_ptr || (m->nnz && (!m->col_ind || !m->val))) return FB_ERR_INVALID;
  if(m->row_ptr[0] != 0 || m->row_ptr[m->rows] != m->nnz) return FB_ERR_INVALID;
  for(uint64_t r = 0; r < m->rows; ++r)
    if(m->row_ptr[r + 1] < m->row_ptr[r]) return FB_ERR_INVALID;
  for(uint64_t i = 0; i < m->nnz; ++i)
    if(m->col_ind[i] >= m->cols) return FB_ERR_INVALID;
  return FB_OK;
}

// SparseMatrixCSR member layout: _elements = {val}, _indices = {col_ind, row_ptr},
// _scalar_index = {rows*columns, rows, columns, used_elements}, _scalar_dt = {0}
// (sparse_matrix_csr.hpp:357-375); the empty matrix has no arrays (:316-324).
Parts csr_parts(const fb_csr_host* m)
{
  Parts p;
  p.scalar_index = {m->rows * m->cols, m->rows, m->cols, m->nnz};
  p.scalar_dt = {0.0};
  if(m->rows > 0) {
    p.elements_size = {m->nnz};
    p.elements = {m->val};
    p.indices_size = {m->nnz, m->rows + 1};
    p.indices = {m->col_ind, m->row_ptr};
  }
  return p;
}

int csr_from_parts(const Parts& p, fb_csr_host* out)
{
  *out = fb_csr_host{};
  if(p.scalar_index.size() < 4) return FB_ERR_FORMAT;
  const uint64_t rows = p.scalar_index[1], cols = p.scalar_index[2], nnz = p.scalar_index[3];
  if(p.elements.empty() && p.indices.empty()) {
    if(rows != 0 || nnz != 0) return FB_ERR_FORMAT;
    out->cols = cols;
    out->row_ptr = alloc_copy<uint64_t>(nullptr, 0);
    out->col_ind = alloc_copy<uint64_t>(nullptr, 0);
    out->val = alloc_copy<double>(nullptr, 0);
    if(!out->row_ptr || !out->col_ind || !out->val) { csr_free(out); return FB_ERR_ALLOC; }
    const_cast<uint64_t*>(out->row_ptr)[0] = 0;
    return FB_OK;
  }
  if(p.elements.size() != 1 || p.indices.size() != 2) return FB_ERR_FORMAT;
  if(p.elements_size[0] != nnz || p.indices_size[0] != nnz || p.indices_size[1] != rows + 1) return FB_ERR_FORMAT;
  out->rows = rows;
  out->cols = cols;
  out->nnz = nnz;
  out->val = alloc_copy<double>(p.elements[0], nnz);
  out->col_ind = alloc_copy<uint64_t>(p.indices[0], nnz);
  out->row_ptr = alloc_copy<uint64_t>(p.indices[1], rows + 1);
  if(!out->row_ptr || !out->col_ind || !out->val) { csr_free(out); return FB_ERR_ALLOC; }
  if(csr_check(out) != FB_OK) { csr_free(out); return FB_ERR_FORMAT; }
  return FB_OK;
}

// DenseVector layout: _elements = {values}, _scalar_index = {size} (dense_vector.hpp:177-220);
// the empty vector has no arrays.
Parts dv_parts(const double* data, uint64_t n)
{
  Parts p;
  p.scalar_index = {n};
  if(n > 0) {
    p.elements_size = {n};
    p.elements = {data};
  }
  return p;
}

int dv_from_parts(const Parts& p, uint64_t* n, double** data)
{
  if(p.scalar_index.empty() || !p.indices.empty()) return FB_ERR_FORMAT;
  const uint64_t size = p.scalar_index[0];
  if(p.elements.empty() ? size != 0 : (p.elements.size() != 1 || p.elements_size[0] != size)) return FB_ERR_FORMAT;
  double* d = alloc_copy<double>(size ? p.elements[0] : nullptr, size);
  if(!d) return FB_ERR_ALLOC;
  *n = size;
  *data = d;
  return FB_OK;
}

// ---------------------------------------------------------------------------------------------
// whole-file helpers
int read_file(const char* path, std::string& s)
{
  if(!path) return FB_ERR_INVALID;
  FILE* f = std::fopen(path, "rb");
  if(!f) return FB_ERR_IO;
  s.clear();
  char chunk[1 << 16];
  size_t got;
  while((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) s.append(chunk, got);
  const bool err = std::ferror(f) != 0;
  std::fclose(f);
  return err ? FB_ERR_IO : FB_OK;
}

// Line cursor over a text buffer; each line is NUL-terminated in place (the line feed is
// overwritten), so strtod/strtol never read into the next line.
struct Lines {
  std::string& s;
  size_t pos = 0;
  explicit Lines(std::string& str) : s(str) {}
  char* next()
  {
    if(pos >= s.size()) return nullptr;
    size_t e = s.find('\n', pos);
    if(e == std::string::npos) e = s.size();
    else s[e] = '\0';
    char* line = &s[pos];
    pos = e + 1;
    return line;
  }
};

bool blank(const char* l)
{
  for(; *l; ++l)
    if(*l != ' ' && *l != '\t' && *l != '\r') return false;
  return true;
}

bool comment(const char* l)
{
  while(*l == ' ' || *l == '\t') ++l;
  return *l == '%';
}

// first line that is neither a comment nor blank (the size line); nullptr at the end
char* size_line(Lines& lines)
{
  char* l;
  while((l = lines.next()) != nullptr)
    if(!comment(l) && !blank(l)) return l;
  return nullptr;
}

// unsigned integer token (atol semantics: leading blanks, optional sign, digits); a
// negative or missing value is a format error
bool parse_index(char*& p, uint64_t& v)
{
  char* e;
  long long x = std::strtoll(p, &e, 10);
  if(e == p || x < 0) return false;
  v = uint64_t(x);
  p = e;
  return true;
}

// "%.6e" of std::scientific at the default precision, independent of the C locale
struct Text {
  std::string buf;
  FILE* f;
  bool ok = true;
  explicit Text(FILE* file) : f(file) { buf.reserve(1 << 20); }
  void flush()
  {
    if(ok && !buf.empty()) ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    buf.clear();
  }
  void str(const char* s) { buf.append(s); }
  void u(uint64_t v)
  {
    char t[24];
    auto r = std::to_chars(t, t + sizeof(t), v);
    buf.append(t, r.ptr);
  }
  void d(double v)
  {
    char t[40];
    auto r = std::to_chars(t, t + sizeof(t), v, std::chars_format::scientific, 6);
    buf.append(t, r.ptr);
  }
  void ch(char c)
  {
    buf.push_back(c);
    if(buf.size() >= (1 << 20)) flush();
  }
};

int open_write(const char* path, bool text, FILE*& f)
{
  if(!path) return FB_ERR_INVALID;
  f = std::fopen(path, text ? "w" : "wb");
  return f ? FB_OK : FB_ERR_IO;
}

int close_write(FILE* f, bool ok)
{
  const bool closed = std::fclose(f) == 0;
  return ok && closed ? FB_OK : FB_ERR_IO;
}

// ---------------------------------------------------------------------------------------------
// MatrixMarket coordinate matrices
int mtx_read_matrix(std::string& s, fb_csr_host* out)
{
  Lines lines(s);
  char* head = lines.next();
  if(!head) return FB_ERR_FORMAT;
  const bool general = std::strstr(head, "%%MatrixMarket matrix coordinate real general") != nullptr;
  const bool symmetric = std::strstr(head, "%%MatrixMarket matrix coordinate real symmetric") != nullptr;
  if(!general && !symmetric) return FB_ERR_FORMAT;
  char* l = size_line(lines);
  uint64_t rows, cols;
  if(!l || !parse_index(l, rows) || !parse_index(l, cols)) return FB_ERR_FORMAT;
  // entries as (row, col, val) triples, symmetric ones mirrored (sparse_matrix_csr.hpp:1198-1203)
  std::vector<uint64_t> er, ec;
  std::vector<double> ev;
  while((l = lines.next()) != nullptr) {
    if(blank(l)) continue;
    uint64_t r, c;
    if(!parse_index(l, r) || !parse_index(l, c)) return FB_ERR_FORMAT;
    if(r < 1 || r > rows || c < 1 || c > cols) return FB_ERR_FORMAT;
    const double v = std::strtod(l, nullptr);
    er.push_back(r - 1); ec.push_back(c - 1); ev.push_back(v);
    if(symmetric && r != c) { er.push_back(c - 1); ec.push_back(r - 1); ev.push_back(v); }
  }
  const uint64_t nnz = er.size();
  // counting sort by row, then each row by column (the reference's map<row, map<col, val>>
  // ordering)
  uint64_t* rp = static_cast<uint64_t*>(std::calloc(rows + 1, sizeof(uint64_t)));
  uint64_t* ci = static_cast<uint64_t*>(std::malloc(std::max<uint64_t>(nnz, 1) * sizeof(uint64_t)));
  double* va = static_cast<double*>(std::malloc(std::max<uint64_t>(nnz, 1) * sizeof(double)));
  *out = fb_csr_host{rows, cols, nnz, rp, ci, va};
  if(!rp || !ci || !va) { csr_free(out); return FB_ERR_ALLOC; }
  for(uint64_t i = 0; i < nnz; ++i) ++rp[er[i] + 1];
  for(uint64_t r = 0; r < rows; ++r) rp[r + 1] += rp[r];
  std::vector<uint64_t> fill(rp, rp + rows);
  for(uint64_t i = 0; i < nnz; ++i) {
    const uint64_t at = fill[er[i]]++;
    ci[at] = ec[i];
    va[at] = ev[i];
  }
  std::vector<std::pair<uint64_t, double>> row;
  for(uint64_t r = 0; r < rows; ++r) {
    const uint64_t b = rp[r], e = rp[r + 1];
    bool sorted = true;
    for(uint64_t i = b + 1; i < e; ++i) {
      if(ci[i] == ci[i - 1]) { csr_free(out); return FB_ERR_FORMAT; }
      sorted &= ci[i] > ci[i - 1];
    }
    if(sorted) continue;
    row.clear();
    for(uint64_t i = b; i < e; ++i) row.emplace_back(ci[i], va[i]);
    // stable: of two equal columns the first in the file comes first (then rejected below)
    std::stable_sort(row.begin(), row.end(),
                     [](const std::pair<uint64_t, double>& x, const std::pair<uint64_t, double>& y) { return x.first < y.first; });
    for(uint64_t i = b; i < e; ++i) {
      ci[i] = row[i - b].first;
      va[i] = row[i - b].second;
      if(i > b && ci[i] == ci[i - 1]) { csr_free(out); return FB_ERR_FORMAT; }
    }
  }
  return FB_OK;
}

int mtx_write_matrix(FILE* f, const fb_csr_host* m, bool symmetric)
{
  Text t(f);
  uint64_t count = m->nnz;
  if(symmetric) {
    count = 0;
    for(uint64_t r = 0; r < m->rows; ++r)
      for(uint64_t i = m->row_ptr[r]; i < m->row_ptr[r + 1]; ++i) count += r >= m->col_ind[i];
  }
  t.str(symmetric ? "%%MatrixMarket matrix coordinate real symmetric\n" : "%%MatrixMarket matrix coordinate real general\n");
  t.u(m->rows); t.ch(' '); t.u(m->cols); t.ch(' '); t.u(count); t.ch('\n');
  for(uint64_t r = 0; r < m->rows; ++r)
    for(uint64_t i = m->row_ptr[r]; i < m->row_ptr[r + 1]; ++i) {
      const uint64_t c = m->col_ind[i];
      if(symmetric && r < c) continue;
      t.u(r + 1); t.ch(' '); t.u(c + 1); t.ch(' '); t.d(m->val[i]); t.ch('\n');
    }
  t.flush();
  return t.ok ? FB_OK : FB_ERR_IO;
}

// ---------------------------------------------------------------------------------------------
// text vectors
int mtx_read_vector(std::string& s, std::vector<double>& v)
{
  Lines lines(s);
  char* head = lines.next();
  if(!head || !std::strstr(head, "%%MatrixMarket matrix array real general")) return FB_ERR_FORMAT;
  char* l = size_line(lines);
  uint64_t rows, cols;
  if(!l || !parse_index(l, rows) || !parse_index(l, cols) || cols != 1) return FB_ERR_FORMAT;
  v.clear();
  // every further line is one value; a blank line reads as atof("") = 0 (dense_vector.hpp:650-664)
  while((l = lines.next()) != nullptr) {
    if(v.size() == rows) return blank(l) && lines.next() == nullptr ? FB_OK : FB_ERR_FORMAT;
    v.push_back(std::strtod(l, nullptr));
  }
  return v.size() == rows ? FB_OK : FB_ERR_FORMAT;
}

int exp_read_vector(std::string& s, std::vector<double>& v)
{
  Lines lines(s);
  v.clear();
  char* l;
  // lines holding '#' are skipped, every other line is one value (dense_vector.hpp:677-699)
  while((l = lines.next()) != nullptr) {
    if(std::strchr(l, '#')) continue;
    v.push_back(std::strtod(l, nullptr));
  }
  return FB_OK;
}

int text_write_vector(FILE* f, const double* data, uint64_t n, bool mtx)
{
  Text t(f);
  if(mtx) {
    t.str("%%MatrixMarket matrix array real general\n");
    t.u(n); t.str(" 1\n");
  }
  for(uint64_t i = 0; i < n; ++i) { t.d(data[i]); t.ch('\n'); }
  t.flush();
  return t.ok ? FB_OK : FB_ERR_IO;
}

// MatrixMarket sparse vectors ("coordinate real general", one column): the Dirichlet list of a
// UnitFilter (SparseVector::read_from / write_out, kernel/lafem/sparse_vector.hpp:517-680).
// Entries come back sorted by index; of repeated indices the last in the file is kept, as the
// reference's sort() keeps it (sparse_vector.hpp:412-470).
int mtx_read_sparse_vector(std::string& s, uint64_t& size, std::vector<uint64_t>& idx, std::vector<double>& val)
{
  Lines lines(s);
  char* head = lines.next();
  if(!head || !std::strstr(head, "%%MatrixMarket matrix coordinate real general")) return FB_ERR_FORMAT;
  char* l = size_line(lines);
  uint64_t rows, cols, nnz;
  if(!l || !parse_index(l, rows) || !parse_index(l, cols) || !parse_index(l, nnz) || cols != 1) return FB_ERR_FORMAT;
  std::vector<std::pair<uint64_t, double>> e;
  while((l = lines.next()) != nullptr) {
    if(blank(l)) continue;
    uint64_t r, c;
    if(!parse_index(l, r) || !parse_index(l, c) || r < 1 || r > rows) return FB_ERR_FORMAT;
    e.emplace_back(r - 1, std::strtod(l, nullptr));
  }
  if(e.size() != nnz) return FB_ERR_FORMAT;
  std::stable_sort(e.begin(), e.end(),
                   [](const std::pair<uint64_t, double>& a, const std::pair<uint64_t, double>& b) { return a.first < b.first; });
  idx.clear();
  val.clear();
  for(size_t i = 0; i < e.size(); ++i) {
    if(i + 1 < e.size() && e[i + 1].first == e[i].first) continue;  // a later entry of the same index
    idx.push_back(e[i].first);
    val.push_back(e[i].second);
  }
  size = rows;
  return FB_OK;
}

}  // namespace

extern "C" {

FB_API int fb_io_csr_read(const char* path, int mode, fb_csr_host* out)
{
  if(!out) return FB_ERR_INVALID;
  *out = fb_csr_host{};
  if(mode != FB_FILE_MTX && mode != FB_FILE_CSR && mode != FB_FILE_BINARY) return FB_ERR_UNSUPPORTED;
  std::string s;
  int rc = read_file(path, s);
  if(rc != FB_OK) return rc;
  if(mode == FB_FILE_MTX) return mtx_read_matrix(s, out);
  Parts p;
  rc = deserialise(s.data(), s.size(), kMagicCsr, p);
  return rc != FB_OK ? rc : csr_from_parts(p, out);
}

FB_API int fb_io_csr_write(const char* path, int mode, const fb_csr_host* m, int symmetric)
{
  if(mode != FB_FILE_MTX && mode != FB_FILE_CSR && mode != FB_FILE_BINARY) return FB_ERR_UNSUPPORTED;
  int rc = csr_check(m);
  if(rc != FB_OK) return rc;
  FILE* f;
  if((rc = open_write(path, mode == FB_FILE_MTX, f)) != FB_OK) return rc;
  if(mode == FB_FILE_MTX) return close_write(f, mtx_write_matrix(f, m, symmetric != 0) == FB_OK);
  Sink s;
  s.f = f;
  serialise(s, csr_parts(m), kMagicCsr);
  return close_write(f, s.ok);
}

FB_API int fb_io_csr_serialised_size(const fb_csr_host* m, uint64_t* size)
{
  const int rc = csr_check(m);
  if(rc != FB_OK || !size) return rc != FB_OK ? rc : FB_ERR_INVALID;
  *size = serialised_size(csr_parts(m));
  return FB_OK;
}

FB_API int fb_io_csr_serialise(const fb_csr_host* m, void* buf, uint64_t capacity)
{
  const int rc = csr_check(m);
  if(rc != FB_OK) return rc;
  if(!buf) return FB_ERR_INVALID;
  const Parts p = csr_parts(m);
  if(serialised_size(p) > capacity) return FB_ERR_TOO_LARGE;
  Sink s;
  s.buf = static_cast<char*>(buf);
  s.cap = capacity;
  serialise(s, p, kMagicCsr);
  return s.ok ? FB_OK : FB_ERR_TOO_LARGE;
}

FB_API int fb_io_csr_deserialise(const void* buf, uint64_t size, fb_csr_host* out)
{
  if(!buf || !out) return FB_ERR_INVALID;
  *out = fb_csr_host{};
  Parts p;
  const int rc = deserialise(static_cast<const char*>(buf), size, kMagicCsr, p);
  return rc != FB_OK ? rc : csr_from_parts(p, out);
}

FB_API void fb_io_csr_release(fb_csr_host* m)
{
  if(m) csr_free(m);
}

FB_API int fb_io_vector_read(const char* path, int mode, uint64_t* n, double** data)
{
  if(!n || !data) return FB_ERR_INVALID;
  *n = 0;
  *data = nullptr;
  if(mode != FB_FILE_EXP && mode != FB_FILE_MTX && mode != FB_FILE_DV && mode != FB_FILE_BINARY)
    return FB_ERR_UNSUPPORTED;
  std::string s;
  int rc = read_file(path, s);
  if(rc != FB_OK) return rc;
  if(mode == FB_FILE_DV || mode == FB_FILE_BINARY) {
    Parts p;
    rc = deserialise(s.data(), s.size(), kMagicDv, p);
    return rc != FB_OK ? rc : dv_from_parts(p, n, data);
  }
  std::vector<double> v;
  rc = mode == FB_FILE_MTX ? mtx_read_vector(s, v) : exp_read_vector(s, v);
  if(rc != FB_OK) return rc;
  double* d = alloc_copy<double>(v.data(), v.size());
  if(!d) return FB_ERR_ALLOC;
  *n = v.size();
  *data = d;
  return FB_OK;
}

FB_API int fb_io_vector_write(const char* path, int mode, const double* data, uint64_t n)
{
  if(mode != FB_FILE_EXP && mode != FB_FILE_MTX && mode != FB_FILE_DV && mode != FB_FILE_BINARY)
    return FB_ERR_UNSUPPORTED;
  if(n && !data) return FB_ERR_INVALID;
  const bool text = mode == FB_FILE_EXP || mode == FB_FILE_MTX;
  FILE* f;
  int rc = open_write(path, text, f);
  if(rc != FB_OK) return rc;
  if(text) return close_write(f, text_write_vector(f, data, n, mode == FB_FILE_MTX) == FB_OK);
  Sink s;
  s.f = f;
  serialise(s, dv_parts(data, n), kMagicDv);
  return close_write(f, s.ok);
}

FB_API int fb_io_vector_serialised_size(uint64_t n, uint64_t* size)
{
  if(!size) return FB_ERR_INVALID;
  *size = serialised_size(dv_parts(nullptr, n));
  return FB_OK;
}

FB_API int fb_io_vector_serialise(const double* data, uint64_t n, void* buf, uint64_t capacity)
{
  if(!buf || (n && !data)) return FB_ERR_INVALID;
  const Parts p = dv_parts(data, n);
  if(serialised_size(p) > capacity) return FB_ERR_TOO_LARGE;
  Sink s;
  s.buf = static_cast<char*>(buf);
  s.cap = capacity;
  serialise(s, p, kMagicDv);
  return s.ok ? FB_OK : FB_ERR_TOO_LARGE;
}

FB_API int fb_io_vector_deserialise(const void* buf, uint64_t size, uint64_t* n, double** data)
{
  if(!buf || !n || !data) return FB_ERR_INVALID;
  *n = 0;
  *data = nullptr;
  Parts p;
  const int rc = deserialise(static_cast<const char*>(buf), size, kMagicDv, p);
  return rc != FB_OK ? rc : dv_from_parts(p, n, data);
}

FB_API int fb_io_sparse_vector_read(const char* path, int mode, uint64_t* size, uint64_t* nnz, uint64_t** indices,
                                    double** values)
{
  if(!size || !nnz || !indices || !values) return FB_ERR_INVALID;
  *size = *nnz = 0;
  *indices = nullptr;
  *values = nullptr;
  if(mode != FB_FILE_MTX) return FB_ERR_UNSUPPORTED;
  std::string s;
  int rc = read_file(path, s);
  if(rc != FB_OK) return rc;
  std::vector<uint64_t> idx;
  std::vector<double> val;
  if((rc = mtx_read_sparse_vector(s, *size, idx, val)) != FB_OK) return rc;
  uint64_t* pi = alloc_copy<uint64_t>(idx.data(), idx.size());
  double* pv = alloc_copy<double>(val.data(), val.size());
  if(!pi || !pv) {
    std::free(pi);
    std::free(pv);
    return FB_ERR_ALLOC;
  }
  *nnz = idx.size();
  *indices = pi;
  *values = pv;
  return FB_OK;
}

FB_API int fb_io_sparse_vector_write(const char* path, int mode, uint64_t size, uint64_t nnz, const uint64_t* indices,
                                     const double* values)
{
  if(mode != FB_FILE_MTX) return FB_ERR_UNSUPPORTED;
  if(nnz && (!indices || !values)) return FB_ERR_INVALID;
  for(uint64_t i = 0; i < nnz; ++i)
    if(indices[i] >= size || (i > 0 && indices[i] <= indices[i - 1])) return FB_ERR_INVALID;
  FILE* f;
  int rc = open_write(path, true, f);
  if(rc != FB_OK) return rc;
  Text t(f);
  t.str("%%MatrixMarket matrix coordinate real general\n");
  t.u(size); t.str(" 1 "); t.u(nnz); t.ch('\n');
  for(uint64_t i = 0; i < nnz; ++i) {
    t.u(indices[i] + 1); t.str(" 1 "); t.d(values[i]); t.ch('\n');
  }
  t.flush();
  return close_write(f, t.ok);
}

FB_API void fb_io_free(void* p)
{
  std::free(p);
}

}  // extern "C"
