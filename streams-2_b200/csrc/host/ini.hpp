// Reader for the solver's INI input files (singleideal.ini, field_info0.dat).
//
// Syntax follows the cfgio parser used by STREAmS-2
// (code/third-party/cfgio/cfgio_mod.F90:776-812 parse_text, :409-466 getters):
//   * a line whose first non-blank character is '#' or ';' is a comment;
//   * "[name]" opens a section;
//   * "key = value" adds a parameter to the current section;
//   * scalar getters use Fortran list-directed semantics: the value is the first
//     token, a token ends at a blank, a comma or a ';' (so "10,controls,x=0" reads 10);
//   * real literals may use a Fortran 'D' exponent (1.0D+04).
// Arrays are comma or blank separated lists, ended by ';'.
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace streams_b200 {

class IniFile {
 public:
  IniFile() = default;
  static IniFile parse_file(const std::string& path);
  static IniFile parse_text(const std::string& text);

  bool has_section(const std::string& sec) const;
  bool has_key(const std::string& sec, const std::string& key) const;
  const std::string& raw(const std::string& sec, const std::string& key) const;

  int get_int(const std::string& sec, const std::string& key) const;
  double get_double(const std::string& sec, const std::string& key) const;
  std::vector<double> get_double_array(const std::string& sec, const std::string& key) const;
  std::vector<int> get_int_array(const std::string& sec, const std::string& key) const;

  int get_int_or(const std::string& sec, const std::string& key, int dflt) const {
    return has_key(sec, key) ? get_int(sec, key) : dflt;
  }
  double get_double_or(const std::string& sec, const std::string& key, double dflt) const {
    return has_key(sec, key) ? get_double(sec, key) : dflt;
  }

  void set(const std::string& sec, const std::string& key, const std::string& val);
  std::string to_text() const;

 private:
  std::vector<std::string> order_;
  std::map<std::string, std::vector<std::pair<std::string, std::string>>> data_;
};

// Thrown for malformed or missing input; the message names the offending key.
struct InputError : public std::runtime_error {
  explicit InputError(const std::string& m) : std::runtime_error(m) {}
};

}  // namespace streams_b200
