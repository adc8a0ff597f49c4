#include "opcode.hpp"

#include <algorithm>
#include <cctype>

namespace lfb {
namespace op {

int arity(int o)
{
    switch (o) {
        case CONSTANT: case VAR_X: case VAR_Y: case VAR_Z: case VAR_FREE:
        case ORACLE:
            return 0;
        case SQUARE: case SQRT: case NEG: case SIN: case COS: case TAN:
        case ASIN: case ACOS: case ATAN: case EXP: case ABS: case LOG:
        case RECIP: case CONST_VAR:
            return 1;
        case ADD: case MUL: case MIN: case MAX: case SUB: case DIV:
        case ATAN2: case POW: case NTH_ROOT: case MOD: case NANFILL:
        case COMPARE:
            return 2;
        default:
            return -1;
    }
}

const char* enum_name(int o)
{
    switch (o) {
        case INVALID: return "INVALID";
        case CONSTANT: return "CONSTANT";
        case VAR_X: return "VAR_X";
        case VAR_Y: return "VAR_Y";
        case VAR_Z: return "VAR_Z";
        case VAR_FREE: return "VAR_FREE";
        case CONST_VAR: return "CONST_VAR";
        case SQUARE: return "SQUARE";
        case SQRT: return "SQRT";
        case NEG: return "NEG";
        case SIN: return "SIN";
        case COS: return "COS";
        case TAN: return "TAN";
        case ASIN: return "ASIN";
        case ACOS: return "ACOS";
        case ATAN: return "ATAN";
        case EXP: return "EXP";
        case ADD: return "ADD";
        case MUL: return "MUL";
        case MIN: return "MIN";
        case MAX: return "MAX";
        case SUB: return "SUB";
        case DIV: return "DIV";
        case ATAN2: return "ATAN2";
        case POW: return "POW";
        case NTH_ROOT: return "NTH_ROOT";
        case MOD: return "MOD";
        case NANFILL: return "NANFILL";
        case ABS: return "ABS";
        case RECIP: return "RECIP";
        case LOG: return "LOG";
        case COMPARE: return "COMPARE";
        case ORACLE: return "ORACLE";
        default: return "";
    }
}

std::string scm_name(int o)
{
    std::string s = enum_name(o);
    for (auto& c : s) {
        c = (c == '_') ? '-' : static_cast<char>(std::tolower(c));
    }
    return s;
}

int from_scm_name(const std::string& s_)
{
    std::string s = s_;
    for (auto& c : s) {
        c = static_cast<char>(std::tolower(c));
    }
    for (int o = 0; o < LAST_OP; ++o) {
        if (scm_name(o) == s) {
            return o;
        }
    }
    return INVALID;
}

std::string op_string(int o)
{
    switch (o) {
        case VAR_X: return "x";
        case VAR_Y: return "y";
        case VAR_Z: return "z";
        case ADD: return "+";
        case MUL: return "*";
        case NEG: case SUB: return "-";
        case RECIP: case DIV: return "/";
        case INVALID: case CONSTANT: case ORACLE: case LAST_OP: return "";
        default: return scm_name(o);
    }
}

bool is_commutative(int o)
{
    return o == ADD || o == MUL || o == MIN || o == MAX;
}

bool is_idempotent(int o)
{
    return o == MIN || o == MAX;
}

}  // namespace op
}  // namespace lfb
