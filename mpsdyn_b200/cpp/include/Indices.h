// shrt::Indices of the reference (src/wrapper/Indices.h): a vector of ints
// with short constructors for up to four dimensions.
#pragma once

#include <initializer_list>
#include <vector>

namespace shrt {

class Indices : public std::vector<int> {
 public:
  Indices() {}
  explicit Indices(int a) : std::vector<int>{a} {}
  Indices(int a, int b) : std::vector<int>{a, b} {}
  Indices(int a, int b, int c) : std::vector<int>{a, b, c} {}
  Indices(int a, int b, int c, int d) : std::vector<int>{a, b, c, d} {}
  Indices(const std::vector<int>& v) : std::vector<int>(v) {}
};

}  // namespace shrt
