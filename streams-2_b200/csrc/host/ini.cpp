#include "ini.hpp"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace streams_b200 {

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

std::string strip_comment(const std::string& v) {
  size_t p = v.find_first_of(";#");
  return trim(p == std::string::npos ? v : v.substr(0, p));
}

// Fortran list-directed tokenisation: separators are blanks and commas.
std::vector<std::string> tokens(const std::string& v) {
  std::vector<std::string> out;
  std::string cur;
  for (char c : strip_comment(v)) {
    if (c == ',' || std::isspace(static_cast<unsigned char>(c))) {
      if (!cur.empty()) out.push_back(cur);
      cur.clear();
    } else {
      cur.push_back(c);
    }
  }
  if (!cur.empty()) out.push_back(cur);
  return out;
}

double to_double(const std::string& tok, const std::string& what) {
  std::string t = tok;
  for (char& c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) throw InputError("cannot read a real from '" + tok + "' (" + what + ")");
  return v;
}

int to_int(const std::string& tok, const std::string& what) {
  char* end = nullptr;
  long v = std::strtol(tok.c_str(), &end, 10);
  if (end == tok.c_str()) throw InputError("cannot read an integer from '" + tok + "' (" + what + ")");
  return static_cast<int>(v);
}

}  // namespace

IniFile IniFile::parse_text(const std::string& text) {
  IniFile ini;
  std::istringstream is(text);
  std::string line, section = "DEFAULTS";
  while (std::getline(is, line)) {
    std::string s = trim(line);
    if (s.empty() || s[0] == '#' || s[0] == ';') continue;
    if (s[0] == '[') {
      size_t e = s.find(']');
      if (e == std::string::npos) throw InputError("Wrong section title: " + s);
      section = trim(s.substr(1, e - 1));
      continue;
    }
    size_t eq = s.find('=');
    if (eq == std::string::npos) continue;
    ini.set(section, trim(s.substr(0, eq)), trim(s.substr(eq + 1)));
  }
  return ini;
}

IniFile IniFile::parse_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw InputError("cannot open input file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_text(ss.str());
}

void IniFile::set(const std::string& sec, const std::string& key, const std::string& val) {
  auto it = data_.find(sec);
  if (it == data_.end()) {
    order_.push_back(sec);
    data_[sec] = {};
    it = data_.find(sec);
  }
  for (auto& kv : it->second)
    if (kv.first == key) {
      kv.second = val;
      return;
    }
  it->second.emplace_back(key, val);
}

bool IniFile::has_section(const std::string& sec) const { return data_.count(sec) > 0; }

bool IniFile::has_key(const std::string& sec, const std::string& key) const {
  auto it = data_.find(sec);
  if (it == data_.end()) return false;
  for (const auto& kv : it->second)
    if (kv.first == key) return true;
  return false;
}

const std::string& IniFile::raw(const std::string& sec, const std::string& key) const {
  auto it = data_.find(sec);
  if (it != data_.end())
    for (const auto& kv : it->second)
      if (kv.first == key) return kv.second;
  throw InputError("missing input key [" + sec + "] " + key);
}

int IniFile::get_int(const std::string& sec, const std::string& key) const {
  auto t = tokens(raw(sec, key));
  if (t.empty()) throw InputError("empty value for [" + sec + "] " + key);
  return to_int(t[0], sec + ":" + key);
}

double IniFile::get_double(const std::string& sec, const std::string& key) const {
  auto t = tokens(raw(sec, key));
  if (t.empty()) throw InputError("empty value for [" + sec + "] " + key);
  return to_double(t[0], sec + ":" + key);
}

std::vector<double> IniFile::get_double_array(const std::string& sec, const std::string& key) const {
  std::vector<double> out;
  for (const auto& t : tokens(raw(sec, key))) out.push_back(to_double(t, sec + ":" + key));
  return out;
}

std::vector<int> IniFile::get_int_array(const std::string& sec, const std::string& key) const {
  std::vector<int> out;
  for (const auto& t : tokens(raw(sec, key))) out.push_back(to_int(t, sec + ":" + key));
  return out;
}

std::string IniFile::to_text() const {
  std::ostringstream os;
  for (const auto& s : order_) {
    os << "[" << s << "]\n";
    for (const auto& kv : data_.at(s)) os << kv.first << " = " << kv.second << "\n";
    os << "\n";
  }
  return os.str();
}

}  // namespace streams_b200
