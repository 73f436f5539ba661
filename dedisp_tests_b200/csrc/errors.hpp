// Error handling shared by the plan classes and the C API.
//
// The C++ layer reports failures by throwing dedisp::Error, a
// std::runtime_error whose message follows the reference format
// "An error occurred within dedisp on line L of F: <error string>"
// (src/common/dedisp_error.hpp:105-121) and which also carries the
// dedisp_error code.
#pragma once

#include <stdexcept>
#include <string>

#include "dedisp.h"

namespace dedisp {

class Error : public std::runtime_error {
public:
    Error(dedisp_error code, const std::string& msg)
        : std::runtime_error(msg), m_code(code) {}
    dedisp_error code() const { return m_code; }

private:
    dedisp_error m_code;
};

[[noreturn]] void throw_error_at(dedisp_error code, const char* file, int line,
                                 const char* detail = nullptr);

}  // namespace dedisp

#define DD_THROW(code) ::dedisp::throw_error_at((code), __FILE__, __LINE__)
#define DD_THROW_MSG(code, msg) \
    ::dedisp::throw_error_at((code), __FILE__, __LINE__, (msg))
#define DD_REQUIRE(cond, code) \
    do {                       \
        if (!(cond)) DD_THROW(code); \
    } while (0)
