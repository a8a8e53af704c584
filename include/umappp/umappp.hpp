#ifndef UMAPPP_UMAPPP_HPP
#define UMAPPP_UMAPPP_HPP

/**
 * @file umappp.hpp
 * @brief Umbrella header of the GPU drop-in for libscran/umappp
 * (include/umappp/umappp.hpp:9-11): Options, Status, initialize() and the
 * stage functions (and the extensions: transform, batched runs, loss and
 * gradient), backed by libumappp_b200.so (C ABI in umapb.h).
 */

#include "Options.hpp"
#include "Status.hpp"
#include "initialize.hpp"
#include "stages.hpp"
#include "transform.hpp"
#include "extensions.hpp"

namespace umappp {}

#endif
