// FieldPatch.hh's serialisation is not used in one process.
#pragma once
namespace boost { namespace serialization { class access; } }
#define BOOST_SERIALIZATION_SPLIT_MEMBER()
