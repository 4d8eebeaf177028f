// Minimal stand-in for gflags (test infrastructure): the reference only names
// the namespace.
#pragma once
namespace gflags {}
