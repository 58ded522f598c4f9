// capi_internal.hpp -- the opaque handle behind include/spaqr_b200.h.
#pragma once
#include <string>

#include "engine.hpp"

struct spq_tree {
  spq::Tree* t;
  std::string err;
};
