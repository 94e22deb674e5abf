// Error plumbing shared by the C-ABI translation units: every entry point turns C++
// exceptions into a status code and a thread-local message.
#pragma once
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/trisk_b200.h"
#include "mesh.hpp"

namespace trisk {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

}  // namespace trisk

#define TRISK_API_BEGIN try {
#define TRISK_API_END                                                  \
  }                                                                    \
  catch (const trisk::Error& e) {                                      \
    trisk::set_last_error(e.what());                                   \
    return e.code;                                                     \
  }                                                                    \
  catch (const trisk::MeshError& e) {                                  \
    trisk::set_last_error(e.what());                                   \
    return TRISK_ERR_MESH;                                             \
  }                                                                    \
  catch (const std::bad_alloc&) {                                      \
    trisk::set_last_error("host allocation failed");                   \
    return TRISK_ERR_ARGUMENT;                                         \
  }                                                                    \
  catch (const std::exception& e) {                                    \
    trisk::set_last_error(e.what());                                   \
    return TRISK_ERR_ARGUMENT;                                         \
  }                                                                    \
  catch (...) {                                                        \
    trisk::set_last_error("unknown error");                            \
    return TRISK_ERR_ARGUMENT;                                         \
  }                                                                    \
  return TRISK_OK;
