// Minimal stand-in for cereal's binary archive header, so that the
// reference's host graph code (include/Graph.h, src/Graph.cpp) compiles
// without the cereal dependency (cereal @ ebef1e9 is fetched at configure
// time by the reference's CMake and is not vendored).  Only the names that
// Graph.h mentions exist; (de)serialisation is not used by the oracle.
#pragma once
#include <iostream>
#include <stdexcept>
#include <string>
namespace cereal {
struct Exception : std::runtime_error {
  explicit Exception(const std::string &what) : std::runtime_error(what) {}
};
struct BinaryInputArchive {
  explicit BinaryInputArchive(std::istream &) {}
  template <class... Ts> void operator()(Ts &&...) {
    throw Exception("cereal stub: deserialisation is not available");
  }
};
struct BinaryOutputArchive {
  explicit BinaryOutputArchive(std::ostream &) {}
  template <class... Ts> void operator()(Ts &&...) {
    throw Exception("cereal stub: serialisation is not available");
  }
};
}  // namespace cereal
