// spiffe_b200/csrc/sdds.cu -- SDDS1 reading and writing for the command
// surface (host code; the layout is described in sdds.hpp).
#include "sdds.hpp"

#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <cstring>

#include "namelist.hpp"

namespace spiffe_sdds {

size_t type_size(Type t)
{
  switch (t) {
  case T_DOUBLE: case T_LONG64: case T_ULONG64: return 8;
  case T_FLOAT: case T_LONG: case T_ULONG: return 4;
  case T_SHORT: case T_USHORT: return 2;
  case T_CHARACTER: return 1;
  default: return 0;
  }
}

static bool parse_type(const std::string &s, Type &t)
{
  static const struct { const char *n; Type t; } names[] = {
    {"double", T_DOUBLE}, {"float", T_FLOAT}, {"long64", T_LONG64}, {"ulong64", T_ULONG64}, {"long", T_LONG},
    {"ulong", T_ULONG}, {"short", T_SHORT}, {"ushort", T_USHORT}, {"string", T_STRING}, {"character", T_CHARACTER}};
  for (const auto &n : names)
    if (s == n.n) {
      t = n.t;
      return true;
    }
  return false;
}

static const char *type_name(Type t)
{
  switch (t) {
  case T_DOUBLE: return "double";
  case T_FLOAT: return "float";
  case T_LONG64: return "long64";
  case T_ULONG64: return "ulong64";
  case T_LONG: return "long";
  case T_ULONG: return "ulong";
  case T_SHORT: return "short";
  case T_USHORT: return "ushort";
  case T_STRING: return "string";
  default: return "character";
  }
}

static double text_number(const std::string &s)
{
  if (s.size() == 1 && !std::isdigit((unsigned char)s[0]))
    return (double)(unsigned char)s[0]; // a character value
  return std::strtod(s.c_str(), nullptr);
}

// ------------------------------------------------------------------ reader

bool Reader::open(const std::string &path, std::string &err)
{
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) {
    err = "unable to open " + path + ": " + std::strerror(errno);
    return false;
  }
  data_.clear();
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0)
    data_.append(buf, n);
  std::fclose(fp);
  if (data_.compare(0, 4, "SDDS") != 0) {
    err = path + " is not an SDDS file";
    return false;
  }
  params_.clear();
  cols_.clear();
  pos_ = data_.find('\n');
  if (pos_ == std::string::npos) {
    err = path + ": truncated header";
    return false;
  }
  pos_++;
  bool big_endian = false, have_data = false;
  int additional = 0;
  std::string pending;
  while (!have_data && pos_ < data_.size()) {
    size_t eol = data_.find('\n', pos_);
    if (eol == std::string::npos)
      eol = data_.size();
    std::string line = data_.substr(pos_, eol - pos_);
    pos_ = eol + 1;
    if (pending.empty()) {
      size_t k = 0;
      while (k < line.size() && std::isspace((unsigned char)line[k]))
        k++;
      if (k < line.size() && line[k] == '!') {
        if (line.find("big-endian") != std::string::npos)
          big_endian = true;
        continue;
      }
      if (k == line.size())
        continue;
    }
    pending += line;
    pending += '\n';
    if (pending.find("&end") == std::string::npos && pending.find("&END") == std::string::npos)
      continue;
    size_t p = 0;
    std::string group, e2;
    std::vector<spiffe_nl::NlEntry> ents;
    while (spiffe_nl::next_block(pending, p, group, ents, e2)) {
      if (group == "parameter" || group == "column") {
        Def d;
        bool typed = false;
        for (const auto &e : ents) {
          if (e.name == "name") d.name = e.value;
          else if (e.name == "units") d.units = e.value;
          else if (e.name == "description") d.description = e.value;
          else if (e.name == "type") typed = parse_type(e.value, d.type);
          else if (e.name == "fixed_value") {
            d.fixed = true;
            d.fixed_value = e.value;
          }
        }
        if (!typed || d.name.empty()) {
          err = path + ": bad &" + group + " definition";
          return false;
        }
        (group == "parameter" ? params_ : cols_).push_back(d);
      } else if (group == "data") {
        for (const auto &e : ents) {
          if (e.name == "mode") {
            if (e.value == "binary")
              binary_ = true;
            else if (e.value == "ascii")
              binary_ = false;
            else {
              err = path + ": unknown data mode " + e.value;
              return false;
            }
          } else if (e.name == "no_row_counts")
            no_row_counts_ = std::atoi(e.value.c_str()) != 0;
          else if (e.name == "column_major_order")
            column_major_ = std::atoi(e.value.c_str()) != 0;
          else if (e.name == "additional_header_lines")
            additional = std::atoi(e.value.c_str());
          else if (e.name == "lines_per_row" && std::atoi(e.value.c_str()) > 1) {
            err = path + ": lines_per_row > 1 is not supported";
            return false;
          }
        }
        have_data = true;
      } else if (group == "array") {
        err = path + ": SDDS arrays are not supported";
        return false;
      }
    }
    if (!e2.empty()) {
      err = path + ": " + e2;
      return false;
    }
    pending.clear();
  }
  if (!have_data) {
    err = path + ": no &data command in the header";
    return false;
  }
  if (!binary_)
    for (int i = 0; i < additional; i++) {
      size_t eol = data_.find('\n', pos_);
      pos_ = eol == std::string::npos ? data_.size() : eol + 1;
    }
  swap_ = big_endian; // this library runs on little-endian hosts only
  return true;
}

int Reader::param_index(const std::string &name) const
{
  for (size_t i = 0; i < params_.size(); i++)
    if (params_[i].name == name)
      return (int)i;
  return -1;
}

int Reader::column_index(const std::string &name) const
{
  for (size_t i = 0; i < cols_.size(); i++)
    if (cols_[i].name == name)
      return (int)i;
  return -1;
}

bool Reader::next_page(Page &p, std::string &err)
{
  err.clear();
  p = Page{};
  p.param_text.resize(params_.size());
  p.param.resize(params_.size());
  for (size_t i = 0; i < params_.size(); i++)
    if (params_[i].fixed) {
      p.param_text[i] = params_[i].fixed_value;
      p.param[i] = text_number(params_[i].fixed_value);
    }
  p.col.resize(cols_.size());
  return binary_ ? read_binary(p, err) : read_ascii(p, err);
}

// splits a line into tokens; double quotes group a token
static void tokens(const std::string &line, std::vector<std::string> &out)
{
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && std::isspace((unsigned char)line[i]))
      i++;
    if (i >= line.size())
      break;
    if (line[i] == '"') {
      size_t e = line.find('"', i + 1);
      if (e == std::string::npos)
        e = line.size();
      out.push_back(line.substr(i + 1, e - i - 1));
      i = e + 1;
    } else {
      size_t e = i;
      while (e < line.size() && !std::isspace((unsigned char)line[e]))
        e++;
      out.push_back(line.substr(i, e - i));
      i = e;
    }
  }
}

bool Reader::read_ascii(Page &p, std::string &err)
{
  auto next_line = [&](std::string &line, bool skip_blank) -> bool {
    while (pos_ < data_.size()) {
      size_t eol = data_.find('\n', pos_);
      if (eol == std::string::npos)
        eol = data_.size();
      line = data_.substr(pos_, eol - pos_);
      pos_ = eol + 1;
      if (!line.empty() && line.back() == '\r')
        line.pop_back();
      size_t k = 0;
      while (k < line.size() && std::isspace((unsigned char)line[k]))
        k++;
      if (k < line.size() && line[k] == '!')
        continue;
      if (k == line.size() && skip_blank)
        continue;
      return true;
    }
    return false;
  };
  std::string line;
  bool started = false;
  for (size_t i = 0; i < params_.size(); i++) {
    if (params_[i].fixed)
      continue;
    if (!next_line(line, true))
      return false; // end of file
    started = true;
    std::vector<std::string> t;
    tokens(line, t);
    std::string v = params_[i].type == T_STRING ? (t.empty() ? "" : (line.find('"') != std::string::npos ? t[0] : line))
                                                : (t.empty() ? "" : t[0]);
    p.param_text[i] = v;
    p.param[i] = text_number(v);
  }
  const size_t nc = cols_.size();
  std::vector<std::string> t;
  if (!no_row_counts_) {
    if (!next_line(line, true)) {
      if (started)
        err = "truncated SDDS page";
      return false;
    }
    const long long rows = std::atoll(line.c_str());
    if (rows < 0) {
      err = "bad SDDS row count";
      return false;
    }
    p.rows = rows;
    for (auto &c : p.col)
      c.reserve((size_t)rows);
    size_t need = (size_t)rows * nc;
    while (t.size() < need) {
      if (!next_line(line, true)) {
        err = "truncated SDDS page";
        return false;
      }
      tokens(line, t);
    }
  } else {
    // rows until a blank line or the end of the file
    bool any = started;
    while (next_line(line, !any)) {
      size_t k = 0;
      while (k < line.size() && std::isspace((unsigned char)line[k]))
        k++;
      if (k == line.size())
        break;
      any = true;
      const size_t before = t.size();
      tokens(line, t);
      if (t.size() - before != nc) {
        err = "SDDS row with the wrong number of values";
        return false;
      }
    }
    if (!any)
      return false;
    p.rows = nc ? (int64_t)(t.size() / nc) : 0;
  }
  for (size_t c = 0; c < nc; c++) {
    if (cols_[c].type == T_STRING)
      continue;
    p.col[c].resize((size_t)p.rows);
    for (int64_t r = 0; r < p.rows; r++)
      p.col[c][(size_t)r] = text_number(t[(size_t)r * nc + c]);
  }
  return true;
}

template <class V> static V load(const char *s, bool swap)
{
  V v;
  if (!swap) {
    std::memcpy(&v, s, sizeof(V));
  } else {
    char b[sizeof(V)];
    for (size_t i = 0; i < sizeof(V); i++)
      b[i] = s[sizeof(V) - 1 - i];
    std::memcpy(&v, b, sizeof(V));
  }
  return v;
}

static double value_at(const char *s, Type t, bool swap)
{
  switch (t) {
  case T_DOUBLE: return load<double>(s, swap);
  case T_FLOAT: return load<float>(s, swap);
  case T_LONG64: return (double)load<int64_t>(s, swap);
  case T_ULONG64: return (double)load<uint64_t>(s, swap);
  case T_LONG: return load<int32_t>(s, swap);
  case T_ULONG: return load<uint32_t>(s, swap);
  case T_SHORT: return load<int16_t>(s, swap);
  case T_USHORT: return load<uint16_t>(s, swap);
  case T_CHARACTER: return (unsigned char)s[0];
  default: return 0;
  }
}

bool Reader::read_binary(Page &p, std::string &err)
{
  if (pos_ + 4 > data_.size())
    return false; // end of file
  const char *d = data_.data();
  auto need = [&](size_t n) {
    if (pos_ + n > data_.size()) {
      err = "truncated SDDS page";
      return false;
    }
    return true;
  };
  int64_t rows = load<int32_t>(d + pos_, swap_);
  pos_ += 4;
  if (rows == INT32_MIN) { // 64-bit row count follows
    if (!need(8))
      return false;
    rows = load<int64_t>(d + pos_, swap_);
    pos_ += 8;
  }
  if (rows < 0) {
    err = "bad SDDS row count";
    return false;
  }
  p.rows = rows;
  for (size_t i = 0; i < params_.size(); i++) {
    if (params_[i].fixed)
      continue;
    if (params_[i].type == T_STRING) {
      if (!need(4))
        return false;
      const int32_t len = load<int32_t>(d + pos_, swap_);
      pos_ += 4;
      if (len < 0 || !need((size_t)len))
        return false;
      p.param_text[i].assign(d + pos_, (size_t)len);
      pos_ += (size_t)len;
      p.param[i] = text_number(p.param_text[i]);
    } else {
      const size_t sz = type_size(params_[i].type);
      if (!need(sz))
        return false;
      p.param[i] = value_at(d + pos_, params_[i].type, swap_);
      p.param_text[i] = params_[i].type == T_CHARACTER ? std::string(1, d[pos_]) : std::to_string(p.param[i]);
      pos_ += sz;
    }
  }
  const size_t nc = cols_.size();
  for (size_t c = 0; c < nc; c++)
    if (cols_[c].type != T_STRING)
      p.col[c].resize((size_t)rows);
  auto one = [&](size_t c, int64_t r) -> bool {
    if (cols_[c].type == T_STRING) {
      if (!need(4))
        return false;
      const int32_t len = load<int32_t>(d + pos_, swap_);
      pos_ += 4;
      if (len < 0 || !need((size_t)len))
        return false;
      pos_ += (size_t)len;
      return true;
    }
    const size_t sz = type_size(cols_[c].type);
    if (!need(sz))
      return false;
    p.col[c][(size_t)r] = value_at(d + pos_, cols_[c].type, swap_);
    pos_ += sz;
    return true;
  };
  if (column_major_) {
    for (size_t c = 0; c < nc; c++)
      for (int64_t r = 0; r < rows; r++)
        if (!one(c, r))
          return false;
  } else {
    for (int64_t r = 0; r < rows; r++)
      for (size_t c = 0; c < nc; c++)
        if (!one(c, r))
          return false;
  }
  return true;
}

bool read_columns(const std::string &path, const std::vector<std::string> &names, std::vector<std::vector<double>> &out,
                  std::string &err)
{
  Reader r;
  if (!r.open(path, err))
    return false;
  std::vector<int> idx;
  for (const auto &n : names) {
    const int i = r.column_index(n);
    if (i < 0) {
      err = path + ": no column " + n;
      return false;
    }
    if (r.columns()[(size_t)i].type == T_STRING) {
      err = path + ": column " + n + " is not numeric";
      return false;
    }
    idx.push_back(i);
  }
  Page p;
  if (!r.next_page(p, err)) {
    if (err.empty())
      err = path + ": no data";
    return false;
  }
  out.clear();
  for (int i : idx)
    out.push_back(p.col[(size_t)i]);
  return true;
}

// ------------------------------------------------------------------ writer

static std::string quoted(const std::string &s)
{
  bool plain = !s.empty();
  for (char c : s)
    if (std::isspace((unsigned char)c) || c == ',' || c == '&' || c == '"' || c == '$')
      plain = false;
  return plain ? s : "\"" + s + "\"";
}

bool Writer::open(const std::string &path, const std::string &text, const std::string &contents,
                  const std::vector<Def> &params, const std::vector<Def> &cols, std::string &err)
{
  close();
  fp_ = std::fopen(path.c_str(), "wb");
  if (!fp_) {
    err = "unable to open " + path + " for writing: " + std::strerror(errno);
    return false;
  }
  params_ = params;
  cols_ = cols;
  std::string h = "SDDS1\n!# little-endian\n";
  if (!text.empty() || !contents.empty()) {
    h += "&description ";
    if (!text.empty())
      h += "text=" + quoted(text) + ", ";
    if (!contents.empty())
      h += "contents=" + quoted(contents) + ", ";
    h += "&end\n";
  }
  auto def = [&](const char *kind, const Def &d) {
    h += std::string("&") + kind + " name=" + quoted(d.name) + ", ";
    if (!d.units.empty())
      h += "units=" + quoted(d.units) + ", ";
    if (!d.description.empty())
      h += "description=" + quoted(d.description) + ", ";
    h += std::string("type=") + type_name(d.type) + ", ";
    if (d.fixed)
      h += "fixed_value=" + quoted(d.fixed_value) + ", ";
    h += "&end\n";
  };
  for (const Def &d : params_)
    def("parameter", d);
  for (const Def &d : cols_)
    def("column", d);
  h += "&data mode=binary, &end\n";
  if (std::fwrite(h.data(), 1, h.size(), fp_) != h.size()) {
    err = "write error on " + path;
    close();
    return false;
  }
  return true;
}

bool Writer::write_page(const std::vector<double> &pv, const std::vector<std::string> &pt, int64_t rows,
                        const std::vector<const void *> &cols, std::string &err)
{
  if (!fp_) {
    err = "SDDS output is not open";
    return false;
  }
  if (cols.size() != cols_.size()) {
    err = "wrong number of SDDS columns";
    return false;
  }
  std::string b;
  if (rows > INT32_MAX) {
    const int32_t flag = INT32_MIN;
    const int64_t r64 = rows;
    b.append((const char *)&flag, 4);
    b.append((const char *)&r64, 8);
  } else {
    const int32_t r32 = (int32_t)rows;
    b.append((const char *)&r32, 4);
  }
  size_t k = 0;
  for (const Def &d : params_) {
    if (d.fixed)
      continue;
    const double v = k < pv.size() ? pv[k] : 0;
    const std::string s = k < pt.size() ? pt[k] : std::string();
    k++;
    switch (d.type) {
    case T_DOUBLE: b.append((const char *)&v, 8); break;
    case T_FLOAT: { const float f = (float)v; b.append((const char *)&f, 4); break; }
    case T_LONG64: { const int64_t x = (int64_t)v; b.append((const char *)&x, 8); break; }
    case T_ULONG64: { const uint64_t x = (uint64_t)v; b.append((const char *)&x, 8); break; }
    case T_LONG: { const int32_t x = (int32_t)v; b.append((const char *)&x, 4); break; }
    case T_ULONG: { const uint32_t x = (uint32_t)v; b.append((const char *)&x, 4); break; }
    case T_SHORT: { const int16_t x = (int16_t)v; b.append((const char *)&x, 2); break; }
    case T_USHORT: { const uint16_t x = (uint16_t)v; b.append((const char *)&x, 2); break; }
    case T_CHARACTER: b.push_back(s.empty() ? (char)v : s[0]); break;
    case T_STRING: {
      const int32_t len = (int32_t)s.size();
      b.append((const char *)&len, 4);
      b.append(s);
      break;
    }
    }
  }
  if (std::fwrite(b.data(), 1, b.size(), fp_) != b.size()) {
    err = "SDDS write error";
    return false;
  }
  // rows interleaved a block at a time
  size_t row_bytes = 0;
  for (const Def &d : cols_) {
    if (d.type == T_STRING) {
      err = "string columns are not written";
      return false;
    }
    row_bytes += type_size(d.type);
  }
  const int64_t block = 1 << 16;
  std::vector<char> buf((size_t)(row_bytes * (size_t)block));
  for (int64_t r0 = 0; r0 < rows; r0 += block) {
    const int64_t n = rows - r0 < block ? rows - r0 : block;
    char *o = buf.data();
    for (int64_t r = r0; r < r0 + n; r++)
      for (size_t c = 0; c < cols_.size(); c++) {
        const size_t sz = type_size(cols_[c].type);
        std::memcpy(o, (const char *)cols[c] + (size_t)r * sz, sz);
        o += sz;
      }
    if (std::fwrite(buf.data(), 1, (size_t)(o - buf.data()), fp_) != (size_t)(o - buf.data())) {
      err = "SDDS write error";
      return false;
    }
  }
  std::fflush(fp_);
  return true;
}

void Writer::close()
{
  if (fp_)
    std::fclose(fp_);
  fp_ = nullptr;
}

} // namespace spiffe_sdds
