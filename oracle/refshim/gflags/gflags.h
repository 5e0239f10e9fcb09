/* Minimal stand-in for gflags, used only to compile the reference's host
 * oracle sources into oracle/_ref (test infrastructure). Flags become plain
 * globals with their default values. */
#pragma once
#include <cstdint>
#include <string>
#define DEFINE_int32(n, v, t) int32_t FLAGS_##n = v
#define DEFINE_int64(n, v, t) int64_t FLAGS_##n = v
#define DEFINE_uint64(n, v, t) uint64_t FLAGS_##n = v
#define DEFINE_bool(n, v, t) bool FLAGS_##n = v
#define DEFINE_double(n, v, t) double FLAGS_##n = v
#define DEFINE_string(n, v, t) std::string FLAGS_##n = v
#define DECLARE_int32(n) extern int32_t FLAGS_##n
#define DECLARE_int64(n) extern int64_t FLAGS_##n
#define DECLARE_uint64(n) extern uint64_t FLAGS_##n
#define DECLARE_bool(n) extern bool FLAGS_##n
#define DECLARE_double(n) extern double FLAGS_##n
#define DECLARE_string(n) extern std::string FLAGS_##n
