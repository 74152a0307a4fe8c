// spiffe_b200/csrc/namelist.hpp -- the namelist text of spiffe input.
//
// spiffe reads its commands and the &po points of a boundary file as
// namelists (spiffe.c:213-215, geometry.c:133-210): "&group name=value,
// ... &end" with '!' comment lines.  The SDDS namelist library that does this
// in the reference is not part of this project, so this header splits the
// text into blocks of (name, value) pairs; callers convert the values.
#pragma once

#include <cctype>
#include <string>
#include <vector>

namespace spiffe_nl {

struct NlEntry {
  std::string name, value;
};

// Splits the text into "&group name=value, ... &end" blocks (a lone '&' also
// ends a block; '!' starts a comment line), lower-casing as geometry.c:137.
inline bool next_block(const std::string &t, size_t &pos, std::string &group, std::vector<NlEntry> &ents, std::string &err)
{
  ents.clear();
  // skip comment lines and find '&'
  while (pos < t.size()) {
    size_t eol = t.find('\n', pos);
    if (eol == std::string::npos)
      eol = t.size();
    size_t p = pos;
    while (p < eol && std::isspace((unsigned char)t[p]))
      p++;
    if (p < eol && t[p] == '!') {
      pos = eol + 1;
      continue;
    }
    const size_t amp = t.find('&', pos);
    if (amp == std::string::npos || amp > eol) {
      pos = eol + 1;
      continue;
    }
    pos = amp + 1;
    break;
  }
  if (pos >= t.size())
    return false;
  size_t p = pos;
  while (p < t.size() && !std::isspace((unsigned char)t[p]) && t[p] != '&')
    p++;
  group = t.substr(pos, p - pos);
  for (auto &c : group)
    c = (char)std::tolower((unsigned char)c);
  for (;;) {
    while (p < t.size() && (std::isspace((unsigned char)t[p]) || t[p] == ','))
      p++;
    if (p >= t.size()) {
      err = "unterminated namelist";
      return false;
    }
    if (t[p] == '&' || t[p] == '$') {
      // "&end" or a lone '&'
      p++;
      if (t.compare(p, 3, "end") == 0 || t.compare(p, 3, "END") == 0)
        p += 3;
      break;
    }
    size_t q = p;
    while (q < t.size() && t[q] != '=' && !std::isspace((unsigned char)t[q]))
      q++;
    std::string name = t.substr(p, q - p);
    for (auto &c : name)
      c = (char)std::tolower((unsigned char)c);
    p = q;
    while (p < t.size() && std::isspace((unsigned char)t[p]))
      p++;
    if (p >= t.size() || t[p] != '=') {
      err = "namelist syntax: expected '=' after " + name;
      return false;
    }
    p++;
    while (p < t.size() && std::isspace((unsigned char)t[p]))
      p++;
    std::string value;
    if (p < t.size() && t[p] == '"') {
      const size_t e = t.find('"', p + 1);
      if (e == std::string::npos) {
        err = "unterminated string";
        return false;
      }
      value = t.substr(p + 1, e - p - 1);
      p = e + 1;
    } else {
      q = p;
      while (q < t.size() && t[q] != ',' && t[q] != '&' && !std::isspace((unsigned char)t[q]))
        q++;
      value = t.substr(p, q - p);
      p = q;
    }
    ents.push_back({name, value});
  }
  pos = p;
  return true;
}

} // namespace spiffe_nl
