// lmc_internal.h -- shared host-side helpers of libluminis_b200 (not installed).
#pragma once
#include <cstdio>
#include <string>

#include "luminis_b200.h"

namespace lmc {

// Thread-local last-error message behind lmc_last_error().
std::string &last_error();

inline lmc_status fail(lmc_status code, const char *msg)
{
  last_error() = msg;
  return code;
}

inline lmc_status fail(lmc_status code, const std::string &msg)
{
  last_error() = msg;
  return code;
}

}  // namespace lmc
