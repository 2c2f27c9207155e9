// The reference's header name for its class, so that code written against
// src/ScatterGatherImpl.hh finds csrst::ScatterGatherImpl with -I<repo>/include/csrst; the class itself
// (same method names, argument order and meaning over the GPU Simulation)
// lives in csrst.hpp.
#pragma once

#include "csrst.hpp"
