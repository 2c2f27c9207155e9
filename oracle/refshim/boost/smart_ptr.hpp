// The one boost name defs.hh needs, for the reference-source check (oracle/refshim/Ippl.h).
#pragma once
#include <memory>
namespace boost {
using std::shared_ptr;
}
