// Device view of a register tape (plain struct shared by host and device code).
#pragma once
#include <cstdint>

#include "tape.hpp"

namespace lfb {

struct DevTape {
    const RegClause* clauses;
    uint32_t n;
    const float* cpool;
    uint32_t n_cpool;
    uint32_t n_const;
    uint32_t n_regs;
    uint32_t n_choices;
    uint8_t root_kind;
    uint16_t root;
};

}  // namespace lfb
