// chasqui_b200 driver — input files in the reference's format (src/params.hpp:1-6):
//
//   [block]
//   key = value      # comment
//
// plus `block.key=value` overrides from the command line. Lookups with a default record the
// default, so the printed table lists every parameter the run used, as the reference does.
#pragma once
#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>

namespace chqd {

class Params {
 public:
  void read_file(const std::string &path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open input file: " + path);
    std::string raw, block;
    while (std::getline(in, raw)) {
      const std::string line = trim(raw.substr(0, raw.find('#')));
      if (line.empty()) continue;
      if (line.size() >= 2 && line.front() == '[' && line.back() == ']') {
        block = trim(line.substr(1, line.size() - 2));
        continue;
      }
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      kv_[block + "." + trim(line.substr(0, eq))] = trim(line.substr(eq + 1));
    }
  }
  void override_with(const std::string &arg) {
    const size_t eq = arg.find('=');
    if (eq == std::string::npos) throw std::runtime_error("bad override: " + arg);
    kv_[trim(arg.substr(0, eq))] = trim(arg.substr(eq + 1));
  }
  bool has(const std::string &b, const std::string &k) const { return kv_.count(b + "." + k) != 0; }
  std::string str(const std::string &b, const std::string &k) const {
    const auto it = kv_.find(b + "." + k);
    if (it == kv_.end()) throw std::runtime_error("missing parameter " + b + "." + k);
    return it->second;
  }
  std::string str(const std::string &b, const std::string &k, const std::string &dflt) {
    return kv_.emplace(b + "." + k, dflt).first->second;
  }
  double real(const std::string &b, const std::string &k) const { return std::stod(str(b, k)); }
  double real(const std::string &b, const std::string &k, double dflt) {
    if (!has(b, k)) kv_[b + "." + k] = fmt(dflt);
    return std::stod(kv_[b + "." + k]);
  }
  int integer(const std::string &b, const std::string &k) const { return std::stoi(str(b, k)); }
  int integer(const std::string &b, const std::string &k, int dflt) {
    if (!has(b, k)) kv_[b + "." + k] = std::to_string(dflt);
    return std::stoi(kv_[b + "." + k]);
  }
  bool boolean(const std::string &b, const std::string &k, bool dflt) {
    std::string v = str(b, k, dflt ? "true" : "false");
    std::transform(v.begin(), v.end(), v.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return v == "true" || v == "1" || v == "yes";
  }
  void print(std::ostream &os) const {
    std::string cur;
    for (const auto &e : kv_) {
      const size_t dot = e.first.find('.');
      const std::string b = e.first.substr(0, dot);
      if (b != cur) {
        os << "[" << b << "]\n";
        cur = b;
      }
      os << "  " << e.first.substr(dot + 1) << " = " << e.second << "\n";
    }
  }

 private:
  static std::string trim(const std::string &s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
  }
  static std::string fmt(double d) {
    std::ostringstream o;
    o.precision(17);
    o << d;
    return o.str();
  }
  std::map<std::string, std::string> kv_;
};

}  // namespace chqd
