// errors.h -- thread-local last-error message behind pgb_last_error().
#pragma once

#include <string>

#include "../../include/pgb.h"

namespace pgb {
void set_error(const std::string& m);
inline pgb_status fail(pgb_status s, const std::string& m) {
    set_error(m);
    return s;
}
}  // namespace pgb
