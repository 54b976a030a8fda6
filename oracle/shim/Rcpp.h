// Minimal stand-in for the one Rcpp facility the reference engine headers use
// (Rcpp::stop, reached from engine/ModelSpecifics.hpp). Written for the oracle
// build only; R is not part of this toolchain.
#pragma once
#include <stdexcept>
#include <string>
namespace Rcpp {
inline void stop(const std::string& message) { throw std::runtime_error(message); }
}  // namespace Rcpp
