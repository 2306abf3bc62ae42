// Forced-include compatibility header for compiling the reference's util/
// sources with a current libstdc++: fixed-width integer types, std::array and
// std::abs for unsigned arguments (the sources call std::abs on every type).
#pragma once
#include <array>
#include <cstdint>
#include <cstdlib>
namespace std {
inline unsigned int abs(unsigned int x) { return x; }
inline unsigned long abs(unsigned long x) { return x; }
inline unsigned char abs(unsigned char x) { return x; }
inline unsigned short abs(unsigned short x) { return x; }
inline bool abs(bool x) { return x; }
}  // namespace std
