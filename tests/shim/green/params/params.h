// Test stand-in for green::params::params: define<T>(name, description, default), operator[]
// returning a value with as<T>(), and set(name, value) for the test driver.  Test infrastructure.
#pragma once
#include <map>
#include <stdexcept>
#include <string>

namespace green::params {

class value {
 public:
  explicit value(std::string s = "") : s_(std::move(s)) {}
  template <typename T>
  T as() const {
    if constexpr (std::is_same_v<T, std::string>) return s_;
    else if constexpr (std::is_integral_v<T>) return (T)std::stoll(s_);
    else return (T)std::stod(s_);
  }

 private:
  std::string s_;
};

class params {
 public:
  template <typename T>
  void define(const std::string& name, const std::string&, const T& def) {
    if constexpr (std::is_same_v<T, std::string>) v_[name] = def;
    else v_[name] = std::to_string(def);
  }
  void set(const std::string& name, const std::string& val) { v_[name] = val; }
  value operator[](const std::string& name) const {
    auto it = v_.find(name);
    if (it == v_.end()) throw std::runtime_error("no parameter " + name);
    return value(it->second);
  }

 private:
  std::map<std::string, std::string> v_;
};

}  // namespace green::params
