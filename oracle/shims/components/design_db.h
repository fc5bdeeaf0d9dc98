// Oracle build shim (test infrastructure only).
// The reference's compiled_block.h includes "components/design_db.h", a header
// that the reference does not ship. Only two names from it are used on the
// solver path: NetUUID (an opaque id built from a string) and PinDirection.
#pragma once
#include <string>
namespace acutesim { namespace components {
struct NetUUID {
    std::string value;
    static NetUUID fromString(const std::string& s) { return NetUUID{s}; }
};
enum class PinDirection { Input, Output, BiDir, Power };
} }
