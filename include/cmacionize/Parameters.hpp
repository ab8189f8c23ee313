/*
 * params.txt surface of the reference driver (testDensitySubGrid_omp.cpp:948-1013):
 * the YAML subset of YAMLDictionary.hpp (indentation nesting, "value unit"
 * strings converted to SI as in UnitConverter.hpp:97-110).  The keys of the
 * plain method are required; the task-runtime capacity keys are accepted.
 */
#ifndef CMACIONIZE_PARAMETERS_HPP
#define CMACIONIZE_PARAMETERS_HPP

#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

class Parameters {
 private:
  std::map<std::string, std::string> _values;

  static std::string trim(const std::string &s) {
    const size_t b = s.find_first_not_of(" \t\r");
    if (b == std::string::npos) return "";
    const size_t e = s.find_last_not_of(" \t\r");
    return s.substr(b, e - b + 1);
  }

  static double unit_factor(const std::string &unit) {
    if (unit.empty() || unit == "m") return 1.;
    if (unit == "cm") return 0.01;
    if (unit == "pc") return 3.086e16;
    if (unit == "kpc") return 3.086e19;
    if (unit == "angstrom") return 1.e-10;
    if (unit == "km") return 1000.;
    throw std::runtime_error("unknown unit \"" + unit + "\"");
  }

  static double physical(const std::string &v) {
    std::istringstream is(v);
    double x;
    std::string unit;
    if (!(is >> x)) throw std::runtime_error("not a number: \"" + v + "\"");
    is >> unit;
    return x * unit_factor(unit);
  }

  static std::vector<std::string> vector_items(const std::string &v) {
    const size_t b = v.find('['), e = v.rfind(']');
    if (b == std::string::npos || e == std::string::npos || e < b)
      throw std::runtime_error("not a vector: \"" + v + "\"");
    std::vector<std::string> out;
    std::stringstream ss(v.substr(b + 1, e - b - 1));
    std::string item;
    while (std::getline(ss, item, ',')) out.push_back(trim(item));
    if (out.size() != 3) throw std::runtime_error("expected 3 components: \"" + v + "\"");
    return out;
  }

 public:
  explicit Parameters(std::istream &in) {
    std::vector<std::pair<size_t, std::string>> stack;
    std::string raw;
    while (std::getline(in, raw)) {
      const std::string line = raw.substr(0, raw.find('#'));
      if (trim(line).empty()) continue;
      const size_t indent = line.find_first_not_of(' ');
      const size_t colon = line.find(':');
      if (colon == std::string::npos) throw std::runtime_error("cannot parse: \"" + raw + "\"");
      const std::string key = trim(line.substr(0, colon));
      const std::string value = trim(line.substr(colon + 1));
      while (!stack.empty() && stack.back().first >= indent) stack.pop_back();
      std::string full;
      for (auto &p : stack) full += p.second + ":";
      full += key;
      if (value.empty()) stack.push_back({indent, key});
      else _values[full] = value;
    }
  }

  static Parameters from_file(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("unable to open parameter file \"" + path + "\"");
    return Parameters(f);
  }

  bool has(const std::string &key) const { return _values.count(key) > 0; }
  const std::string &get_string(const std::string &key) const {
    auto it = _values.find(key);
    if (it == _values.end()) throw std::runtime_error("missing parameter \"" + key + "\"");
    return it->second;
  }
  double get_physical(const std::string &key) const { return physical(get_string(key)); }
  double get_double(const std::string &key) const { return std::strtod(get_string(key).c_str(), nullptr); }
  unsigned long get_unsigned(const std::string &key) const {
    const double v = get_double(key);
    if (v < 0 || v != (double)(unsigned long)v)
      throw std::runtime_error("not an unsigned integer: " + key);
    return (unsigned long)v;
  }
  bool get_bool(const std::string &key) const {
    const std::string v = get_string(key);
    if (v == "true" || v == "yes" || v == "1") return true;
    if (v == "false" || v == "no" || v == "0") return false;
    throw std::runtime_error("not a boolean: " + key);
  }
  void get_physical_vector(const std::string &key, double out[3]) const {
    const auto items = vector_items(get_string(key));
    for (int a = 0; a < 3; ++a) out[a] = physical(items[a]);
  }
  void get_int_vector(const std::string &key, int out[3]) const {
    const auto items = vector_items(get_string(key));
    for (int a = 0; a < 3; ++a) out[a] = (int)std::strtod(items[a].c_str(), nullptr);
  }
};

/* read_parameters (testDensitySubGrid_omp.cpp:948-1013): the plain-method keys. */
struct PlainMethodParameters {
  double box[6];
  double reemission_probability;
  int ncell[3], num_subgrid[3];
  unsigned int num_photon, number_of_iterations, number_of_sources;
  bool random_density;

  explicit PlainMethodParameters(const Parameters &p) {
    p.get_physical_vector("box:anchor", box);
    p.get_physical_vector("box:sides", box + 3);
    reemission_probability = p.get_double("reemission_probability");
    p.get_int_vector("ncell", ncell);
    p.get_int_vector("num_subgrid", num_subgrid);
    num_photon = (unsigned int)p.get_unsigned("num_photon");
    number_of_iterations = (unsigned int)p.get_unsigned("number_of_iterations");
    number_of_sources = (unsigned int)p.get_unsigned("number_of_sources");
    random_density = p.get_bool("random_density");
    for (int a = 0; a < 3; ++a)
      if (num_subgrid[a] <= 0 || ncell[a] % num_subgrid[a])
        throw std::runtime_error("ncell must be a multiple of num_subgrid");
  }
};

#endif
