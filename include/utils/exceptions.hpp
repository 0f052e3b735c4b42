// exceptions.hpp -- status handling of the C++ drop-in API over
// libpeasoup_b200 (replaces ErrorChecker, reference
// include/utils/exceptions.hpp:13-153).  A failed call throws
// std::runtime_error with the library's message, as the reference did; no
// device-wide synchronisation is implied.
#pragma once
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include "peasoup_b200.h"

class ErrorChecker {
public:
    static void check(int status, const std::string& where)
    {
        if (status == PSX_OK) return;
        std::stringstream msg;
        msg << where << " failed: " << psx_status_string(status);
        const char* detail = psx_last_error();
        if (detail && *detail) msg << " (" << detail << ")";
        throw std::runtime_error(msg.str());
    }

    static void throw_error(const std::string& msg) { throw std::runtime_error(msg); }

    static void check_file_error(std::ifstream& in, const std::string& name)
    {
        if (!in.good()) throw std::runtime_error("File " + name + " could not be opened");
    }
};
