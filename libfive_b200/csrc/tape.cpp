#include "tape.hpp"

#include <algorithm>
#include <queue>

namespace lfb {

bool build_slot_tape(const Tree& root_, SlotTape& out, std::string* err)
{
    const Tree root = root_.optimized();   // flattened: no remap / apply left
    std::vector<uint32_t> kid_pos;
    const auto flat = root.walk(&kid_pos);

    // Slot ids count down from flat.size() so that the root lands on 1
    // (deck.cpp:24-58); slot 0 is the reference's placeholder.  The node at
    // position j of the walk takes slot flat.size() - j.
    const uint32_t n_flat = static_cast<uint32_t>(flat.size());
    uint32_t id = n_flat;
    std::vector<SlotClause> rev;
    rev.reserve(flat.size());
    const Node* axes[3] = {Tree::X().get(), Tree::Y().get(), Tree::Z().get()};
    uint32_t axis_slot[3] = {0, 0, 0};
    for (uint32_t j = 0; j < n_flat; ++j) {
        const Node* m = flat[j];
        auto slot_of_kid = [&](int i) { return n_flat - kid_pos[2 * j + i]; };
        switch (m->kind) {
            case Kind::Constant:
                out.constants.push_back({id, m->value});
                break;
            case Kind::Nullary:
                if (m->op == op::VAR_FREE) {
                    out.vars.push_back({id, m});
                } else if (m->op != op::VAR_X && m->op != op::VAR_Y &&
                           m->op != op::VAR_Z) {
                    if (err) *err = "unsupported nullary opcode";
                    return false;
                }
                break;
            case Kind::Unary:
                rev.push_back({m->op, id, slot_of_kid(0), 0});
                break;
            case Kind::Binary:
                rev.push_back({m->op, id, slot_of_kid(0), slot_of_kid(1)});
                break;
            default:
                if (err) *err = "tree contains an unsupported node";
                return false;
        }
        for (int a = 0; a < 3; ++a) {
            if (m == axes[a]) axis_slot[a] = id;
        }
        --id;
    }
    out.clauses.assign(rev.rbegin(), rev.rend());

    // Axes that the tree does not use take the next free slots, in x, y, z
    // order.
    uint32_t next = n_flat + 1;
    for (int a = 0; a < 3; ++a) {
        if (!axis_slot[a]) axis_slot[a] = next++;
    }
    out.num_clauses = next - 1;
    out.X = axis_slot[0];
    out.Y = axis_slot[1];
    out.Z = axis_slot[2];
    std::sort(out.vars.begin(), out.vars.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    out.root = 1;   // the walk ends at the root
    return true;
}

bool build_reg_tape(const SlotTape& st, RegTape& out, std::string* err)
{
    out = RegTape();
    const uint32_t n_slots = st.num_clauses + 1;

    // Operand descriptor for every slot: kind + index.
    std::vector<uint8_t> kind(n_slots, 0xff);
    std::vector<uint32_t> index(n_slots, 0);
    kind[st.X] = OPND_REG; index[st.X] = 0;
    kind[st.Y] = OPND_REG; index[st.Y] = 1;
    kind[st.Z] = OPND_REG; index[st.Z] = 2;
    for (const auto& c : st.constants) {
        kind[c.first] = OPND_CONST;
        index[c.first] = static_cast<uint32_t>(out.cpool.size());
        out.cpool.push_back(c.second);
    }
    out.n_const = static_cast<uint32_t>(out.cpool.size());
    for (const auto& v : st.vars) {
        kind[v.first] = OPND_VAR;
        index[v.first] = static_cast<uint32_t>(out.cpool.size());
        out.cpool.push_back(0.0f);
        out.var_nodes.push_back(v.second);
        out.var_slots.push_back(v.first);
    }
    out.n_vars = static_cast<uint32_t>(st.vars.size());
    if (out.cpool.size() > 0xffff) {
        if (err) *err = "too many constants and variables for a device tape";
        return false;
    }

    // Evaluation order is the slot tape reversed.
    const size_t n = st.clauses.size();
    std::vector<const SlotClause*> order(n);
    for (size_t i = 0; i < n; ++i) {
        order[i] = &st.clauses[n - 1 - i];
    }

    // Last position at which each slot is read (the root stays live to the
    // end of the tape).
    std::vector<int64_t> last_use(n_slots, -1);
    for (size_t i = 0; i < n; ++i) {
        const auto* c = order[i];
        const int ar = op::arity(c->op);
        if (ar >= 1) last_use[c->a] = static_cast<int64_t>(i);
        if (ar >= 2) last_use[c->b] = static_cast<int64_t>(i);
    }
    last_use[st.root] = static_cast<int64_t>(n);

    std::priority_queue<uint32_t, std::vector<uint32_t>, std::greater<uint32_t>>
        free_regs;
    uint32_t next_reg = 3;
    out.clauses.reserve(n);
    for (size_t i = 0; i < n; ++i) {
        const auto* c = order[i];
        const int ar = op::arity(c->op);
        if (ar < 1) {
            if (err) *err = "unsupported opcode in tape";
            return false;
        }
        RegClause rc{};
        rc.op = static_cast<uint8_t>(c->op);
        auto operand = [&](uint32_t s, uint16_t& idx, int shift) {
            if (kind[s] == 0xff) {
                return false;
            }
            idx = static_cast<uint16_t>(index[s]);
            rc.kinds |= static_cast<uint8_t>(kind[s] << shift);
            return true;
        };
        if (!operand(c->a, rc.a, 0) ||
            (ar == 2 && !operand(c->b, rc.b, 2))) {
            if (err) *err = "tape refers to an undefined slot";
            return false;
        }
        // Release operand registers whose last use is this clause (before
        // allocating the output, which may then reuse one of them).
        auto release = [&](uint32_t s) {
            if (kind[s] == OPND_REG && index[s] >= 3 &&
                last_use[s] == static_cast<int64_t>(i)) {
                free_regs.push(index[s]);
                last_use[s] = -2;   // released once even if read twice
            }
        };
        release(c->a);
        if (ar == 2) release(c->b);

        uint32_t r;
        if (!free_regs.empty()) {
            r = free_regs.top();
            free_regs.pop();
        } else {
            r = next_reg++;
        }
        if (r > 0xffff) {
            if (err) *err = "register file overflow";
            return false;
        }
        rc.out = static_cast<uint16_t>(r);
        kind[c->id] = OPND_REG;
        index[c->id] = r;
        if (c->op == op::MIN || c->op == op::MAX) {
            out.n_choices++;
        }
        out.clauses.push_back(rc);
    }
    out.n_regs = next_reg;
    if (kind[st.root] == 0xff) {
        if (err) *err = "root slot undefined";
        return false;
    }
    out.root_kind = kind[st.root];
    out.root = static_cast<uint16_t>(index[st.root]);
    return true;
}

bool build_wide_list(const RegTape& t, std::vector<WideEntry>& out,
                     uint32_t& root_slot, std::string* err)
{
    const size_t n = t.clauses.size();
    // Register -> slot of the value it holds, walking the tape in order.
    std::vector<uint32_t> slot_of(std::max<uint32_t>(t.n_regs, 3), 0);
    for (uint32_t r = 0; r < 3; ++r) slot_of[r] = r;
    std::vector<uint32_t> level(n + 3, 0);
    std::vector<WideEntry> tmp(n);
    uint32_t max_level = 0;
    for (size_t c = 0; c < n; ++c) {
        const RegClause& rc = t.clauses[c];
        const uint8_t ka = rc.kinds & 3, kb = (rc.kinds >> 2) & 3;
        const bool binary = op::arity(rc.op) == 2;
        WideEntry e{};
        e.a = ka == OPND_REG ? slot_of[rc.a] : rc.a;
        e.b = (binary && kb == OPND_REG) ? slot_of[rc.b] : (binary ? rc.b : 0u);
        uint32_t lv = 0;
        if (ka == OPND_REG) lv = std::max(lv, level[e.a]);
        if (binary && kb == OPND_REG) lv = std::max(lv, level[e.b]);
        ++lv;
        if (lv > kWideMaxLevel) {
            if (err) *err = "tape dependency chain longer than 262143 clauses";
            return false;
        }
        max_level = std::max(max_level, lv);
        const uint32_t kinds = binary ? (rc.kinds & 0xf) : (rc.kinds & 3);
        e.head = rc.op | (kinds << 8) | (WIDE_BOTH << 12) | (lv << kWideLevelShift);
        e.c = static_cast<uint32_t>(c);
        level[3 + c] = lv;
        tmp[c] = e;
        slot_of[rc.out] = static_cast<uint32_t>(3 + c);
    }
    // Counting sort by level, stable in clause order; then operands and the
    // root are renamed from clause slots to list slots.
    std::vector<uint32_t> start(max_level + 2, 0);
    for (size_t c = 0; c < n; ++c) ++start[level[3 + c] + 1];
    for (uint32_t l = 1; l < start.size(); ++l) start[l] += start[l - 1];
    std::vector<uint32_t> pos(n);
    out.assign(n, WideEntry{});
    for (size_t c = 0; c < n; ++c) {
        pos[c] = start[level[3 + c]]++;
        out[pos[c]] = tmp[c];
    }
    for (WideEntry& e : out) {
        const uint32_t kinds = (e.head >> 8) & 0xf;
        const bool binary = op::arity(e.head & 0xff) == 2;
        if ((kinds & 3) == OPND_REG && e.a >= 3) e.a = 3 + pos[e.a - 3];
        if (binary && ((kinds >> 2) & 3) == OPND_REG && e.b >= 3) e.b = 3 + pos[e.b - 3];
    }
    root_slot = t.root_kind == OPND_REG ? slot_of[t.root] : t.root;
    if (t.root_kind == OPND_REG && root_slot >= 3) root_slot = 3 + pos[root_slot - 3];
    return true;
}

}  // namespace lfb
