// spiffe_b200/csrc/sdds.hpp -- the SDDS file layout spiffe reads and writes.
//
// spiffe's input tables (antenna waveforms, antenna.c:88-101; cathode time
// profiles, cathode.c:152-166; saved fields, load_fields.c:56-118) and its
// outputs (screens, screens.c:81-100; field saves, field_saving.c:67-119) are
// SDDS files.  The SDDS library is not part of this project, so this module
// reads and writes the published SDDS1 layout itself: a text header of
// &description / &parameter / &column / &data namelists, then pages in ASCII
// or binary.  Binary pages hold a 32-bit row count, the values of the
// parameters that have no fixed_value, and the rows (row by row, or column
// by column when the header says column_major_order=1).  Arrays (&array) are
// not supported.  Files are written binary, little-endian, row-major, one
// page per write_page call.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace spiffe_sdds {

enum Type { T_DOUBLE, T_FLOAT, T_LONG64, T_ULONG64, T_LONG, T_ULONG, T_SHORT, T_USHORT, T_STRING, T_CHARACTER };

struct Def {
  std::string name, units, description;
  Type type = T_DOUBLE;
  bool fixed = false;     // parameter with fixed_value (not stored per page)
  std::string fixed_value;
};

// One page: parameter values (as text and as numbers, in header order) and
// the numeric columns converted to double (string columns are left empty).
struct Page {
  std::vector<std::string> param_text;
  std::vector<double> param;
  std::vector<std::vector<double>> col;
  int64_t rows = 0;
};

class Reader {
public:
  // Reads the header; false with `err` set if the file is missing or not SDDS.
  bool open(const std::string &path, std::string &err);
  // Next page; false at the end of the file (err empty) or on an error.
  bool next_page(Page &p, std::string &err);
  int param_index(const std::string &name) const;
  int column_index(const std::string &name) const;
  const std::vector<Def> &params() const { return params_; }
  const std::vector<Def> &columns() const { return cols_; }

private:
  bool read_ascii(Page &p, std::string &err);
  bool read_binary(Page &p, std::string &err);
  std::string data_;
  size_t pos_ = 0;
  std::vector<Def> params_, cols_;
  bool binary_ = false, swap_ = false, column_major_ = false, no_row_counts_ = false;
};

class Writer {
public:
  Writer() = default;
  // one owner per open file: moves hand the file over, copies are not allowed
  Writer(const Writer &) = delete;
  Writer &operator=(const Writer &) = delete;
  Writer(Writer &&o) noexcept : fp_(o.fp_), params_(std::move(o.params_)), cols_(std::move(o.cols_)) { o.fp_ = nullptr; }
  Writer &operator=(Writer &&o) noexcept
  {
    if (this != &o) {
      close();
      fp_ = o.fp_;
      params_ = std::move(o.params_);
      cols_ = std::move(o.cols_);
      o.fp_ = nullptr;
    }
    return *this;
  }
  ~Writer() { close(); }
  // Writes the header (the &description's text and contents may be empty);
  // `params` with fixed=true carry their value there.
  bool open(const std::string &path, const std::string &text, const std::string &contents,
            const std::vector<Def> &params, const std::vector<Def> &cols, std::string &err);
  // One page: the values of the non-fixed parameters (numbers, or text for
  // string/character parameters) and one pointer per column to `rows`
  // values of that column's type (double, int32_t for long, int16_t for short).
  bool write_page(const std::vector<double> &param_values, const std::vector<std::string> &param_text, int64_t rows,
                  const std::vector<const void *> &cols, std::string &err);
  void close();
  bool is_open() const { return fp_ != nullptr; }

private:
  FILE *fp_ = nullptr;
  std::vector<Def> params_, cols_;
};

// A whole numeric column of the first page of a file (the form spiffe reads
// waveforms and profiles in).
bool read_columns(const std::string &path, const std::vector<std::string> &names,
                  std::vector<std::vector<double>> &out, std::string &err);

size_t type_size(Type t);

} // namespace spiffe_sdds
