// Shared definitions of the B200 DD-PCG library (host and device).
#pragma once
#include <cstdint>
#include <cstddef>
#include <stdexcept>
#include <string>

#include "../../include/hdd.h"

namespace hdd {

// Reference cell flags (SPGRID_MULTIGRID_FLAGS.h:13-30).
enum : uint32_t {
    F_ACTIVE = 0x00010000u,
    F_DIRICHLET = 0x00020000u,
    F_BOUNDARY = 0x00040000u,
    F_INTERFACE = 0x00080000u,
    F_FACE_MX = 0x00100000u,
    F_FACES = 0x03f00000u,
};

// Compact device flags.  Level 0 (uint16): bits 0-5 face bits in the
// reference order (-x,+x,-y,+y,-z,+z), bit 6 Active, bit 7 Interface,
// bit 8 Boundary.  Coarse levels (uint8): bits 0-5 faces, bit 6 Active,
// bit 7 Boundary.
enum : uint32_t {
    C_FACES = 0x3fu,
    C_ACTIVE = 0x40u,
    C_INTERFACE = 0x80u,
    C_BOUNDARY16 = 0x100u,
    C_BOUNDARY8 = 0x80u,
};

inline uint16_t compact16(uint32_t f) {
    uint16_t c = (uint16_t)((f >> 20) & 0x3fu);
    if (f & F_ACTIVE) c |= C_ACTIVE;
    if (f & F_INTERFACE) c |= C_INTERFACE;
    if (f & F_BOUNDARY) c |= C_BOUNDARY16;
    return c;
}
inline uint8_t compact8(uint32_t f) {
    uint8_t c = (uint8_t)((f >> 20) & 0x3fu);
    if (f & F_ACTIVE) c |= C_ACTIVE;
    if (f & F_BOUNDARY) c |= C_BOUNDARY8;
    return c;
}

struct Error : std::runtime_error {
    hdd_status status;
    Error(hdd_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

}  // namespace hdd
