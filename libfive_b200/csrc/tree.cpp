#include "tree.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <optional>
#include <sstream>
#include <stack>
#include <unordered_map>
#include <unordered_set>
#include <variant>

#include "flat_map.hpp"
#include "scalar_ops.h"

namespace lfb {

static std::atomic<uint64_t> g_serial{1};

////////////////////////////////////////////////////////////////////////////////
// Reference counting

Tree::~Tree()
{
    if (!p) {
        return;
    }
    if (p->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) {
        return;
    }
    // Iterative teardown so that deep chains do not overflow the stack
    // (same reason as libfive/src/tree/tree.cpp:27-69).  The pending list
    // lives on the stack until it outgrows 64 entries.
    const Node* local[64];
    size_t n_local = 0;
    std::vector<const Node*> spill;
    local[n_local++] = p;
    while (n_local || !spill.empty()) {
        const Node* n;
        if (!spill.empty()) {
            n = spill.back();
            spill.pop_back();
        } else {
            n = local[--n_local];
        }
        for (auto k : n->kid) {
            if (k && k->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) {
                if (n_local < 64) {
                    local[n_local++] = k;
                } else {
                    spill.push_back(k);
                }
            }
        }
        delete n;
    }
}

Tree& Tree::operator=(const Tree& o)
{
    Tree tmp(o);
    std::swap(p, tmp.p);
    optimized_flag = o.optimized_flag;
    return *this;
}

Tree& Tree::operator=(Tree&& o) noexcept
{
    std::swap(p, o.p);
    optimized_flag = o.optimized_flag;
    return *this;
}

const Node* Tree::release()
{
    const Node* out = p;
    p = nullptr;
    return out;
}

Tree Tree::reclaim(const Node* n)
{
    return Tree(n, false, false);
}

int Tree::op() const
{
    switch (p->kind) {
        case Kind::Constant: return op::CONSTANT;
        case Kind::Nullary:
        case Kind::Unary:
        case Kind::Binary: return p->op;
        default: return op::INVALID;
    }
}

////////////////////////////////////////////////////////////////////////////////
// Construction

static uint32_t compute_flags(Kind k, int o, const Node* const* kids)
{
    switch (k) {
        case Kind::Nullary:
            return (o == op::VAR_X || o == op::VAR_Y || o == op::VAR_Z)
                ? Node::HAS_XYZ : 0;
        case Kind::Unary:
            return kids[0]->flags;
        case Kind::Binary:
            return kids[0]->flags | kids[1]->flags;
        case Kind::Remap:
            return kids[0]->flags | kids[1]->flags | kids[2]->flags |
                   kids[3]->flags | Node::HAS_REMAP;
        case Kind::Apply:
            return kids[0]->flags | kids[1]->flags | kids[2]->flags |
                   Node::HAS_REMAP;
        default:
            return 0;
    }
}

Tree Tree::make(Kind k, int o, float value, const Node* a, const Node* b,
                const Node* c, const Node* d)
{
    Node* n = new Node;
    n->kind = k;
    n->op = o;
    n->value = value;
    n->kid[0] = a;
    n->kid[1] = b;
    n->kid[2] = c;
    n->kid[3] = d;
    for (auto kk : n->kid) {
        if (kk) kk->refs.fetch_add(1, std::memory_order_relaxed);
    }
    n->flags = compute_flags(k, o, n->kid);
    n->serial = g_serial.fetch_add(1, std::memory_order_relaxed);
    // The node is not shared yet: its one reference (the returned handle's)
    // needs no read-modify-write.
    n->refs.store(1, std::memory_order_relaxed);
    return Tree(n, false, false);
}

Tree Tree::constant(double v)
{
    return make(Kind::Constant, op::CONSTANT, static_cast<float>(v),
                nullptr, nullptr);
}

Tree Tree::X()
{
    static Tree x = make(Kind::Nullary, op::VAR_X, 0, nullptr, nullptr);
    return x;
}
Tree Tree::Y()
{
    static Tree y = make(Kind::Nullary, op::VAR_Y, 0, nullptr, nullptr);
    return y;
}
Tree Tree::Z()
{
    static Tree z = make(Kind::Nullary, op::VAR_Z, 0, nullptr, nullptr);
    return z;
}
Tree Tree::invalid()
{
    static Tree i = make(Kind::Invalid, op::INVALID, 0, nullptr, nullptr);
    return i;
}
Tree Tree::one()
{
    static Tree o = make(Kind::Constant, op::CONSTANT, 1.0f, nullptr, nullptr);
    return o;
}
Tree Tree::var()
{
    return nullary(op::VAR_FREE);
}

Tree Tree::nullary(int o)
{
    if (op::arity(o) != 0) {
        return invalid();
    }
    switch (o) {
        case op::VAR_X: return X();
        case op::VAR_Y: return Y();
        case op::VAR_Z: return Z();
        default: break;
    }
    return make(Kind::Nullary, o, 0, nullptr, nullptr);
}

float fold_constant(int o, float a, float b)
{
    switch (o) {
        case op::ADD: return a + b;
        case op::MUL: return a * b;
        case op::MIN: return sc_min(a, b);
        case op::MAX: return sc_max(a, b);
        case op::SUB: return a - b;
        case op::DIV: return a / b;
        case op::ATAN2: return atan2f(a, b);
        case op::POW: return powf(a, b);
        case op::NTH_ROOT: return sc_nth_root(a, b);
        case op::MOD: return sc_mod(a, b);
        case op::NANFILL: return sc_isnan(a) ? b : a;
        case op::COMPARE: return sc_compare(a, b);
        case op::SQUARE: return a * a;
        case op::SQRT: return sqrtf(a);
        case op::NEG: return -a;
        case op::SIN: return sinf(a);
        case op::COS: return cosf(a);
        case op::TAN: return tanf(a);
        case op::ASIN: return asinf(a);
        case op::ACOS: return acosf(a);
        case op::ATAN: return atanf(a);
        case op::LOG: return logf(a);
        case op::EXP: return expf(a);
        case op::ABS: return fabsf(a);
        case op::RECIP: return 1.0f / a;
        case op::CONST_VAR: return a;
        default: return NAN;
    }
}

// Local simplifications follow tree.cpp:95-123.
Tree Tree::unary(int o, const Tree& a)
{
    return unary_n(o, a.p);
}

Tree Tree::unary_n(int o, const Node* a)
{
    if (op::arity(o) != 1) {
        return invalid();
    }
    if (a->kind == Kind::Constant) {
        return constant(fold_constant(o, a->value, 0.0f));
    }
    if (o == op::ABS) {
        if (a->kind == Kind::Unary &&
            (a->op == op::ABS || a->op == op::SQUARE)) {
            return Tree(a);
        }
    } else if (o == op::NEG) {
        if (a->kind == Kind::Unary && a->op == op::NEG) {
            return Tree(a->kid[0]);
        }
    }
    return make(Kind::Unary, o, 0, a, nullptr);
}

/// Tree::op() of a bare node.
static int op_of(const Node* n)
{
    switch (n->kind) {
        case Kind::Constant: return op::CONSTANT;
        case Kind::Nullary:
        case Kind::Unary:
        case Kind::Binary: return n->op;
        default: return op::INVALID;
    }
}

// Local simplifications follow tree.cpp:141-230, including the exact
// if / else-if chains (e.g. for ADD, a constant lhs stops the search even
// when it is non-zero).
Tree Tree::binary(int o, const Tree& a, const Tree& b)
{
    return binary_n(o, a.p, b.p);
}

Tree Tree::binary_n(int o, const Node* a, const Node* b)
{
    if (op::arity(o) != 2) {
        return invalid();
    }
    const bool ac = a->kind == Kind::Constant;
    const bool bc = b->kind == Kind::Constant;
    if (op_of(a) == op::CONSTANT && op_of(b) == op::CONSTANT) {
        return constant(fold_constant(o, a->value, b->value));
    }
    auto is_neg = [](const Node* t) {
        return t->kind == Kind::Unary && t->op == op::NEG;
    };
    if (o == op::DIV) {
        if (bc && b->value == 1.0f) {
            return Tree(a);
        }
    } else if (o == op::ADD) {
        if (ac) {
            if (a->value == 0.0f) return Tree(b);
        } else if (bc) {
            if (b->value == 0.0f) return Tree(a);
        } else if (a->kind == Kind::Unary) {
            if (a->op == op::NEG) return binary_n(op::SUB, b, a->kid[0]);
        } else if (b->kind == Kind::Unary) {
            if (b->op == op::NEG) return binary_n(op::SUB, a, b->kid[0]);
        }
    } else if (o == op::SUB) {
        if (ac) {
            if (a->value == 0.0f) return unary_n(op::NEG, b);
        } else if (bc) {
            if (b->value == 0.0f) return Tree(a);
        } else if (is_neg(b)) {
            return binary_n(op::ADD, a, b->kid[0]);
        }
    } else if (o == op::MUL) {
        if (ac) {
            if (a->value == 0) return Tree(a);
            if (a->value == 1) return Tree(b);
            if (a->value == -1) return unary_n(op::NEG, b);
        } else if (bc) {
            if (b->value == 0) return Tree(b);
            if (b->value == 1) return Tree(a);
            if (b->value == -1) return unary_n(op::NEG, a);
        } else if (a == b) {
            return unary_n(op::SQUARE, a);
        }
    } else if (o == op::NTH_ROOT || o == op::POW) {
        if (bc && b->value == 1.0f) {
            return Tree(a);
        }
    } else if (o == op::MIN || o == op::MAX) {
        if (a == b) {
            return Tree(a);
        }
    }
    return make(Kind::Binary, o, 0, a, b);
}

Tree operator+(const Tree& a, const Tree& b) { return Tree::binary(op::ADD, a, b); }
Tree operator-(const Tree& a, const Tree& b) { return Tree::binary(op::SUB, a, b); }
Tree operator*(const Tree& a, const Tree& b) { return Tree::binary(op::MUL, a, b); }
Tree operator/(const Tree& a, const Tree& b) { return Tree::binary(op::DIV, a, b); }
Tree operator-(const Tree& a) { return Tree::unary(op::NEG, a); }

////////////////////////////////////////////////////////////////////////////////
// Remap / apply / flatten (tree.cpp:366-528)

Tree Tree::remap(const Tree& x, const Tree& y, const Tree& z) const
{
    if (x == X() && y == Y() && z == Z()) {
        return *this;
    }
    if (p->flags & Node::HAS_XYZ) {
        return make(Kind::Remap, op::INVALID, 0, x.p, y.p, z.p, p);
    }
    return *this;
}

Tree Tree::apply(const Tree& v, const Tree& value) const
{
    if (v.op() != op::VAR_FREE) {
        return invalid();
    }
    return make(Kind::Apply, op::INVALID, 0, v.p, value.p, p);
}

Tree Tree::flatten() const
{
    if (!(p->flags & Node::HAS_REMAP)) {
        return *this;
    }
    using Map = std::unordered_map<const Node*, Tree>;
    using MapPtr = std::shared_ptr<Map>;
    struct Task {
        bool down;
        const Node* t;
        MapPtr m;
    };
    std::vector<Task> todo{{true, p, nullptr}};
    std::vector<Tree> out;

    while (!todo.empty()) {
        Task k = todo.back();
        todo.pop_back();
        auto lookup = [&](const Node* t) {
            if (k.m) {
                auto it = k.m->find(t);
                if (it != k.m->end()) {
                    return it->second;
                }
            }
            return Tree(t);
        };
        if (k.down) {
            switch (k.t->kind) {
                case Kind::Nullary:
                    out.push_back(lookup(k.t));
                    break;
                case Kind::Unary:
                    todo.push_back({false, k.t, k.m});
                    todo.push_back({true, k.t->kid[0], k.m});
                    break;
                case Kind::Binary:
                    todo.push_back({false, k.t, k.m});
                    todo.push_back({true, k.t->kid[0], k.m});
                    todo.push_back({true, k.t->kid[1], k.m});
                    break;
                case Kind::Constant:
                case Kind::Invalid:
                    out.push_back(Tree(k.t));
                    break;
                case Kind::Remap:
                    todo.push_back({false, k.t, k.m});
                    todo.push_back({true, k.t->kid[2], k.m});
                    todo.push_back({true, k.t->kid[1], k.m});
                    todo.push_back({true, k.t->kid[0], k.m});
                    break;
                case Kind::Apply:
                    todo.push_back({false, k.t, k.m});
                    todo.push_back({true, k.t->kid[1], k.m});
                    break;
            }
        } else {
            switch (k.t->kind) {
                case Kind::Unary: {
                    Tree a = std::move(out.back());
                    out.pop_back();
                    out.push_back(a.p != k.t->kid[0] ? unary(k.t->op, a)
                                                     : Tree(k.t));
                    break;
                }
                case Kind::Binary: {
                    Tree a = std::move(out.back());
                    out.pop_back();
                    Tree b = std::move(out.back());
                    out.pop_back();
                    out.push_back((a.p != k.t->kid[0] || b.p != k.t->kid[1])
                                      ? binary(k.t->op, a, b)
                                      : Tree(k.t));
                    break;
                }
                case Kind::Remap: {
                    auto m = std::make_shared<Map>(k.m ? *k.m : Map());
                    (*m)[Z().p] = out.back(); out.pop_back();
                    (*m)[Y().p] = out.back(); out.pop_back();
                    (*m)[X().p] = out.back(); out.pop_back();
                    todo.push_back({true, k.t->kid[3], m});
                    break;
                }
                case Kind::Apply: {
                    auto m = std::make_shared<Map>(k.m ? *k.m : Map());
                    (*m)[k.t->kid[0]] = out.back();
                    out.pop_back();
                    todo.push_back({true, k.t->kid[2], m});
                    break;
                }
                default:
                    break;
            }
        }
    }
    return out.back();
}

////////////////////////////////////////////////////////////////////////////////
// Topological walk (tree.cpp:530-594)

std::vector<const Node*> Tree::walk() const
{
    if (p->flags & Node::HAS_REMAP) {
        return flatten().walk();
    }
    return walk(nullptr);
}

std::vector<const Node*> Tree::walk(std::vector<uint32_t>* kid_pos) const
{
    // Pass 1 gives every distinct node a dense index (one hash lookup per
    // edge of the DAG) and counts its parents; pass 2 emits a node once all
    // its parents are out, through the dense arrays alone, and reversing
    // that order puts every child before its parents (tree.cpp:530-594).
    static std::atomic<size_t> count_hint{1024};   // capacity hint, as in optimized()
    FlatMap<const Node*, uint32_t, PtrHash> index(count_hint.load(std::memory_order_relaxed));
    std::vector<const Node*> nodes{p};
    std::vector<uint32_t> parents{0};
    std::vector<uint32_t> kids{UINT32_MAX, UINT32_MAX};   // 2 per index
    nodes.reserve(count_hint.load(std::memory_order_relaxed) + 1);
    index.emplace(p, 0u);
    auto nkids = [](const Node* n) {
        return n->kind == Kind::Unary ? 1 : n->kind == Kind::Binary ? 2 : 0;
    };
    std::vector<uint32_t> todo{0};
    while (!todo.empty()) {
        const uint32_t ni = todo.back();
        todo.pop_back();
        const Node* n = nodes[ni];
        for (int i = 0; i < nkids(n); ++i) {
            const auto r = index.emplace(n->kid[i], static_cast<uint32_t>(nodes.size()));
            const uint32_t ki = *r.first;
            if (r.second) {
                nodes.push_back(n->kid[i]);
                parents.push_back(0);
                kids.push_back(UINT32_MAX);
                kids.push_back(UINT32_MAX);
                todo.push_back(ki);
            }
            kids[2 * ni + i] = ki;
            ++parents[ki];
        }
    }
    const size_t total = nodes.size();
    std::vector<uint32_t> order;   // indices, root first
    order.reserve(total);
    todo.push_back(0);
    while (!todo.empty()) {
        const uint32_t ni = todo.back();
        todo.pop_back();
        order.push_back(ni);
        for (int i = 0; i < 2; ++i) {
            const uint32_t ki = kids[2 * ni + i];
            if (ki != UINT32_MAX && --parents[ki] == 0) {
                todo.push_back(ki);
            }
        }
    }
    count_hint.store(std::max<size_t>(1024, total), std::memory_order_relaxed);
    std::vector<const Node*> flat(total);
    std::vector<uint32_t> pos(kid_pos ? total : 0);
    for (size_t j = 0; j < total; ++j) {
        const uint32_t ni = order[total - 1 - j];
        flat[j] = nodes[ni];
        if (kid_pos) pos[ni] = static_cast<uint32_t>(j);
    }
    if (kid_pos) {
        kid_pos->assign(2 * total, UINT32_MAX);
        for (size_t j = 0; j < total; ++j) {
            const uint32_t ni = order[total - 1 - j];
            for (int i = 0; i < 2; ++i) {
                const uint32_t ki = kids[2 * ni + i];
                if (ki != UINT32_MAX) (*kid_pos)[2 * j + i] = pos[ki];
            }
        }
    }
    return flat;
}

size_t Tree::size() const
{
    std::unordered_set<const Node*> seen;
    std::vector<const Node*> todo{p};
    while (!todo.empty()) {
        const Node* n = todo.back();
        todo.pop_back();
        if (!seen.insert(n).second) {
            continue;
        }
        for (auto k : n->kid) {
            if (k) todo.push_back(k);
        }
    }
    return seen.size();
}

////////////////////////////////////////////////////////////////////////////////
// Optimizer (tree.cpp:612-961)

namespace {

/// Structural key used for deduplication (libfive/include/libfive/tree/key.hpp
/// and TreeData::key in libfive/src/tree/data.cpp).  Constants compare by
/// float value (so +0 and -0 share a key), NaN constants share one key, and
/// every free variable is its own key.
struct Key {
    uint8_t tag;   // 0 invalid, 1 nan, 2 float, 3 nullary, 4 unary/var,
                   // 5 binary, 6 remap, 7 apply
    int op;
    float value;
    const Node* p[4];

    bool operator==(const Key& o) const
    {
        if (tag != o.tag) return false;
        switch (tag) {
            case 0: case 1: return true;
            case 2: return value == o.value;
            case 3: return op == o.op;
            case 4: return op == o.op && p[0] == o.p[0];
            case 5: return op == o.op && p[0] == o.p[0] && p[1] == o.p[1];
            default:
                return p[0] == o.p[0] && p[1] == o.p[1] && p[2] == o.p[2] &&
                       p[3] == o.p[3];
        }
    }
};

struct KeyHash {
    size_t operator()(const Key& k) const
    {
        size_t h = k.tag * 0x9e3779b97f4a7c15ull;
        auto mix = [&](size_t v) {
            h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        };
        switch (k.tag) {
            case 2: {
                const float v = (k.value == 0.0f) ? 0.0f : k.value;
                uint32_t bits;
                std::memcpy(&bits, &v, 4);
                mix(bits);
                break;
            }
            case 3: mix(k.op); break;
            case 4: mix(k.op); mix(reinterpret_cast<size_t>(k.p[0])); break;
            case 5:
                mix(k.op);
                mix(reinterpret_cast<size_t>(k.p[0]));
                mix(reinterpret_cast<size_t>(k.p[1]));
                break;
            default:
                for (auto q : k.p) mix(reinterpret_cast<size_t>(q));
        }
        return h;
    }
};

Key key_of(const Node* n)
{
    Key k{};
    switch (n->kind) {
        case Kind::Constant:
            if (std::isnan(n->value)) {
                k.tag = 1;
            } else {
                k.tag = 2;
                k.value = n->value;
            }
            break;
        case Kind::Nullary:
            if (n->op == op::VAR_FREE) {
                k.tag = 4;
                k.op = n->op;
                k.p[0] = n;
            } else {
                k.tag = 3;
                k.op = n->op;
            }
            break;
        case Kind::Unary:
            k.tag = 4;
            k.op = n->op;
            k.p[0] = n->kid[0];
            break;
        case Kind::Binary:
            k.tag = 5;
            k.op = n->op;
            k.p[0] = n->kid[0];
            k.p[1] = n->kid[1];
            break;
        case Kind::Remap:
            k.tag = 6;
            for (int i = 0; i < 4; ++i) k.p[i] = n->kid[i];
            break;
        case Kind::Apply:
            k.tag = 7;
            for (int i = 0; i < 3; ++i) k.p[i] = n->kid[i];
            break;
        case Kind::Invalid:
            k.tag = 0;
            break;
    }
    return k;
}

/// The optimizer's table of canonical nodes: one reference to each, keyed by
/// the node's structure (key_of).  Slots are bare node pointers (8 bytes,
/// against 64 for a (Key, Tree) pair) probed through a dense one-byte tag
/// array, so that the table of a model of some 10^4-10^5 nodes stays in the
/// host's L2 cache; a slot's node is read only when its tag matches.
class CanonSet {
public:
    explicit CanonSet(size_t expected)
    {
        size_t cap = 16;
        while (cap < 2 * expected) cap <<= 1;
        reset(cap);
    }
    ~CanonSet()
    {
        for (size_t i = 0; i < slots_.size(); ++i) {
            if (tags_[i]) Tree::reclaim(slots_[i]);
        }
    }
    CanonSet(const CanonSet&) = delete;
    CanonSet& operator=(const CanonSet&) = delete;

    size_t size() const { return count_; }

    /// The stored node structurally equal to n; when there is none, n itself,
    /// stored without taking a reference (*inserted = true: the caller hands
    /// the table one).
    const Node* intern(const Node* n, bool* inserted)
    {
        if ((count_ + 1) * 2 > slots_.size()) grow();
        const Key k = key_of(n);
        const uint64_t h = static_cast<uint64_t>(KeyHash()(k)) * 0x9e3779b97f4a7c15ull;
        const uint8_t t = static_cast<uint8_t>((h >> 8) | 1);
        size_t i = static_cast<size_t>(h >> shift_) & mask_;
        while (tags_[i]) {
            if (tags_[i] == t && (slots_[i] == n || key_of(slots_[i]) == k)) {
                *inserted = false;
                return slots_[i];
            }
            i = (i + 1) & mask_;
        }
        tags_[i] = t;
        slots_[i] = n;
        ++count_;
        *inserted = true;
        return n;
    }

    /// The stored constant whose key is v's (every NaN one key, +0 and -0
    /// one key), or null: lets a caller skip building a constant node that
    /// intern() would only find already present.
    const Node* find_constant(float v) const
    {
        Key k{};
        if (std::isnan(v)) {
            k.tag = 1;
        } else {
            k.tag = 2;
            k.value = v;
        }
        const uint64_t h = static_cast<uint64_t>(KeyHash()(k)) * 0x9e3779b97f4a7c15ull;
        const uint8_t t = static_cast<uint8_t>((h >> 8) | 1);
        size_t i = static_cast<size_t>(h >> shift_) & mask_;
        while (tags_[i]) {
            if (tags_[i] == t && key_of(slots_[i]) == k) return slots_[i];
            i = (i + 1) & mask_;
        }
        return nullptr;
    }

private:
    void reset(size_t cap)
    {
        slots_.assign(cap, nullptr);
        tags_.assign(cap, 0);
        mask_ = cap - 1;
        shift_ = 64;
        for (size_t c = cap; c > 1; c >>= 1) --shift_;
        count_ = 0;
    }
    void grow()
    {
        std::vector<const Node*> old_slots;
        std::vector<uint8_t> old_tags;
        old_slots.swap(slots_);
        old_tags.swap(tags_);
        reset(old_slots.size() * 2);
        for (size_t i = 0; i < old_slots.size(); ++i) {
            if (!old_tags[i]) continue;
            const uint64_t h = static_cast<uint64_t>(KeyHash()(key_of(old_slots[i]))) *
                               0x9e3779b97f4a7c15ull;
            size_t j = static_cast<size_t>(h >> shift_) & mask_;
            while (tags_[j]) j = (j + 1) & mask_;
            tags_[j] = old_tags[i];
            slots_[j] = old_slots[i];
            ++count_;
        }
    }

    std::vector<const Node*> slots_;
    std::vector<uint8_t> tags_;
    size_t mask_ = 0;
    unsigned shift_ = 64;
    size_t count_ = 0;
};

/// Orders trees the way the reference orders them by address: here by the
/// creation serial number.
bool serial_less(const Node* a, const Node* b)
{
    return a->serial < b->serial;
}

}  // namespace

Tree Tree::optimized() const
{
    if (optimized_flag) {
        return *this;
    }
    if (p->flags & Node::HAS_REMAP) {
        return flatten().optimized();
    }

    // `canonical` owns one reference to every tree this pass hands around;
    // everything below it (the output stack, affine terms, commutative
    // lists) holds plain pointers, which stay valid because each of them
    // is either a node of the input tree or a canonical entry.
    // Sized from the previous call (a capacity hint only: trees built
    // repeatedly from the same kind of model skip the rehashing).
    static std::atomic<size_t> canon_hint{1024};
    CanonSet canonical(canon_hint.load(std::memory_order_relaxed));
    auto uniq_new = [&canonical](Tree&& t) -> const Node* {
        bool inserted = false;
        const Node* c = canonical.intern(t.get(), &inserted);
        if (inserted) t.release();   // the table keeps t's reference
        return c;
    };
    // uniq_new(constant(v)) without building the node when the table
    // already holds an equal constant (the skipped node would only have
    // taken a creation serial, which orders nothing that survives).
    auto uniq_const = [&canonical, &uniq_new](float v) -> const Node* {
        if (const Node* c = canonical.find_constant(v)) return c;
        return uniq_new(constant(v));
    };
    auto uniq_old = [&canonical](const Node* n) -> const Node* {
        bool inserted = false;
        const Node* c = canonical.intern(n, &inserted);
        if (inserted) Tree(n).release();   // one new reference, for the table
        return c;
    };
    // The constant 1 is created on first use, like the reference's static
    // (tree.cpp:251-254); its creation serial orders it among affine terms,
    // so it must not be touched any earlier than the reference would.
    const Node* one_p = nullptr;
    auto ONE = [&one_p]() {
        if (!one_p) one_p = one().p;
        return one_p;
    };

    // One frame per DOWN task: the affine accumulator (tree -> scale factor)
    // and the commutative list that the reference keeps on two parallel
    // stacks of optionals.  Frames are pooled, so their buffers are reused.
    struct Frame {
        bool has_affine = false;
        bool has_comm = false;
        int comm_op = 0;
        std::vector<std::pair<const Node*, float>> terms;
        FlatMap<const Node*, uint32_t, PtrHash> index{16};
        std::vector<const Node*> list;

        void reset()
        {
            has_affine = has_comm = false;
            terms.clear();
            index.clear();
            list.clear();
        }
        // Adds s to the scale of t.  Terms are looked up by a linear scan
        // while there are few of them, then through `index`.
        void add(const Node* t, float s)
        {
            if (terms.size() < 16) {
                for (auto& e : terms) {
                    if (e.first == t) {
                        e.second += s;
                        return;
                    }
                }
                terms.push_back({t, s});
                if (terms.size() == 16) {
                    for (uint32_t i = 0; i < 16; ++i) {
                        index.emplace(terms[i].first, i);
                    }
                }
                return;
            }
            auto r = index.emplace(t, static_cast<uint32_t>(terms.size()));
            if (r.second) {
                terms.push_back({t, s});
            } else {
                terms[*r.first].second += s;
            }
        }
    };
    std::vector<Frame> frames(1);
    size_t depth = 1;
    auto push_frame = [&]() {
        if (depth == frames.size()) {
            frames.emplace_back();
        } else {
            frames[depth].reset();
        }
        ++depth;
    };

    struct Task {
        enum { DOWN, UP, UP_AFFINE, UP_COMM } type;
        const Node* t;
        float scale;
    };
    std::vector<Task> todo{{Task::DOWN, p, 1.0f}};
    std::vector<const Node*> out;
    std::vector<std::pair<const Node*, float>> pos, neg;

    auto deliver = [&](const Node* self, float scale) {
        Frame& f = frames[depth - 1];
        if (f.has_affine) {
            if (self->kind == Kind::Constant) {
                f.add(ONE(), scale * self->value);
            } else {
                f.add(self, scale);
            }
        } else if (f.has_comm) {
            f.list.push_back(self);
        } else {
            out.push_back(self);
        }
    };

    while (!todo.empty()) {
        const Task task = todo.back();
        todo.pop_back();

        if (task.type == Task::DOWN) {
            const Node* d = task.t;
            todo.push_back({Task::UP, d, task.scale});
            push_frame();

            // Either turns this frame into an affine / commutative
            // accumulator, or (when the parent frame already accumulates
            // the same thing) drops it so that the children feed the
            // parent's accumulator directly.
            bool marked_affine = false;
            auto mark_affine = [&]() {
                todo.pop_back();
                if (!frames[depth - 2].has_affine) {
                    frames[depth - 1].has_affine = true;
                    todo.push_back({Task::UP_AFFINE, nullptr, 0.0f});
                } else {
                    --depth;
                }
                marked_affine = true;
            };
            auto mark_comm = [&](int o) {
                todo.pop_back();
                const Frame& parent = frames[depth - 2];
                if (!parent.has_comm || parent.comm_op != o) {
                    frames[depth - 1].has_comm = true;
                    frames[depth - 1].comm_op = o;
                    todo.push_back({Task::UP_COMM, nullptr, task.scale});
                } else {
                    --depth;
                }
            };

            if (d->kind == Kind::Unary) {
                if (d->op == op::NEG) {
                    mark_affine();
                    todo.push_back({Task::DOWN, d->kid[0], -task.scale});
                }
            } else if (d->kind == Kind::Binary) {
                const Node* l = d->kid[0];
                const Node* r = d->kid[1];
                if (d->op == op::ADD) {
                    mark_affine();
                    todo.push_back({Task::DOWN, l, task.scale});
                    todo.push_back({Task::DOWN, r, task.scale});
                } else if (d->op == op::SUB) {
                    mark_affine();
                    todo.push_back({Task::DOWN, l, task.scale});
                    todo.push_back({Task::DOWN, r, -task.scale});
                } else if (d->op == op::MUL) {
                    if (l->kind == Kind::Constant) {
                        mark_affine();
                        todo.push_back({Task::DOWN, r, l->value * task.scale});
                    } else if (r->kind == Kind::Constant) {
                        mark_affine();
                        todo.push_back({Task::DOWN, l, r->value * task.scale});
                    } else {
                        mark_comm(op::MUL);
                    }
                } else if (d->op == op::DIV) {
                    if (r->kind == Kind::Constant) {
                        mark_affine();
                        todo.push_back({Task::DOWN, l, task.scale / r->value});
                    }
                } else if (d->op == op::MIN || d->op == op::MAX) {
                    mark_comm(d->op);
                }
            }

            if (!marked_affine) {
                if (d->kind == Kind::Unary) {
                    todo.push_back({Task::DOWN, d->kid[0], 1.0f});
                } else if (d->kind == Kind::Binary) {
                    todo.push_back({Task::DOWN, d->kid[0], 1.0f});
                    todo.push_back({Task::DOWN, d->kid[1], 1.0f});
                }
            }
        } else if (task.type == Task::UP) {
            --depth;
            const Node* d = task.t;
            // The reference enters d in the table before replacing it when
            // an operand changed (tree.cpp:776-789); that entry can never be
            // found again (no node built later has d's old operands, which
            // only ever come out of this pass changed), so it is skipped.
            const Node* self = nullptr;
            if (d->kind == Kind::Unary) {
                const Node* a = out.back();
                out.pop_back();
                self = a != d->kid[0] ? uniq_new(unary_n(d->op, a)) : uniq_old(d);
            } else if (d->kind == Kind::Binary) {
                const Node* a = out.back();
                out.pop_back();
                const Node* b = out.back();
                out.pop_back();
                self = (a != d->kid[0] || b != d->kid[1]) ? uniq_new(binary_n(d->op, a, b))
                                                          : uniq_old(d);
            } else {
                self = uniq_old(d);
            }
            deliver(self, task.scale);
        } else if (task.type == Task::UP_AFFINE) {
            // Nothing below pushes a frame, so the popped frame's buffers
            // stay valid while they are read.
            const Frame& f = frames[depth - 1];
            --depth;

            // Split into positive and negative terms; NaN scales go with the
            // positive terms and zero scales are dropped (tree.cpp:832-848).
            pos.clear();
            neg.clear();
            for (const auto& kv : f.terms) {
                const float s = kv.second;
                if (s > 0.0f) {
                    pos.push_back({kv.first, s});
                } else if (s < 0.0f) {
                    neg.push_back({kv.first, -s});
                } else if (s != 0.0f) {
                    pos.push_back({kv.first, s});
                }
            }
            // Ascending scale, then creation order.  NaN scales sort last:
            // the reference compares them with `<` alone, which is not a
            // strict weak order, so its placement of NaN terms depends on
            // hash-table iteration order and is not reproducible anyway.
            auto order = [](const std::pair<const Node*, float>& a,
                            const std::pair<const Node*, float>& b) {
                const bool an = std::isnan(a.second);
                const bool bn = std::isnan(b.second);
                if (an != bn) {
                    return bn;
                }
                if (!an && a.second != b.second) {
                    return a.second < b.second;
                }
                return serial_less(a.first, b.first);
            };
            std::sort(pos.begin(), pos.end(), order);
            std::sort(neg.begin(), neg.end(), order);

            auto collapse = [&](const std::vector<std::pair<const Node*, float>>& v) {
                const Node* acc = nullptr;
                size_t i = 0;
                while (i < v.size()) {
                    const float mult = v[i].second;
                    const Node* t = v[i].first;
                    ++i;
                    while (i < v.size() && v[i].second == mult) {
                        t = uniq_new(binary_n(op::ADD, t, v[i].first));
                        ++i;
                    }
                    if (mult != 1) {
                        if (t == ONE()) {
                            t = uniq_const(mult);
                        } else {
                            t = uniq_new(binary_n(op::MUL, t,
                                                  uniq_const(mult)));
                        }
                    }
                    acc = acc ? uniq_new(binary_n(op::ADD, acc, t)) : t;
                }
                return acc ? acc : uniq_const(0.0f);
            };
            const Node* P = collapse(pos);
            const Node* N = collapse(neg);
            const Node* self = uniq_new(binary_n(op::SUB, P, N));
            Frame& parent = frames[depth - 1];
            if (parent.has_comm) {
                parent.list.push_back(self);
            } else {
                out.push_back(self);
            }
        } else {  // UP_COMM
            Frame& f = frames[depth - 1];
            --depth;
            std::sort(f.list.begin(), f.list.end(), serial_less);
            auto end = f.list.end();
            if (op::is_idempotent(f.comm_op)) {
                end = std::unique(f.list.begin(), f.list.end());
            }
            const Node* self = f.list.front();
            for (auto it = f.list.begin() + 1; it != end; ++it) {
                self = uniq_new(binary_n(f.comm_op, self, *it));
            }
            deliver(self, task.scale);
        }
    }
    canon_hint.store(std::max<size_t>(1024, canonical.size()), std::memory_order_relaxed);
    return Tree(out.back(), true, true);
}

////////////////////////////////////////////////////////////////////////////////
// Printing (tree.cpp:269-337)

void Tree::print(std::ostream& s) const
{
    struct Item {
        const Node* n;
        char c;
    };
    std::vector<Item> todo{{p, 0}};
    std::vector<int> ops{op::INVALID};
    while (!todo.empty()) {
        Item it = todo.back();
        todo.pop_back();
        if (!it.n) {
            switch (it.c) {
                case ')': s << ')'; ops.pop_back(); break;
                case '|': ops.pop_back(); break;
                case ' ': s << ' '; break;
            }
            continue;
        }
        const Node* n = it.n;
        switch (n->kind) {
            case Kind::Nullary:
                s << op::op_string(n->op);
                break;
            case Kind::Unary:
                s << "(" << op::op_string(n->op) << " ";
                ops.push_back(n->op);
                todo.push_back({nullptr, ')'});
                todo.push_back({n->kid[0], 0});
                break;
            case Kind::Binary:
                if (op::is_commutative(n->op) && ops.back() == n->op) {
                    todo.push_back({nullptr, '|'});
                } else {
                    s << "(" << op::op_string(n->op) << " ";
                    todo.push_back({nullptr, ')'});
                }
                ops.push_back(n->op);
                todo.push_back({n->kid[1], 0});
                todo.push_back({nullptr, ' '});
                todo.push_back({n->kid[0], 0});
                break;
            case Kind::Constant:
                s << n->value;
                break;
            case Kind::Remap:
                s << "(remap ";
                todo.push_back({nullptr, ')'});
                ops.push_back(op::INVALID);
                todo.push_back({n->kid[2], 0});
                todo.push_back({nullptr, ' '});
                todo.push_back({n->kid[1], 0});
                todo.push_back({nullptr, ' '});
                todo.push_back({n->kid[0], 0});
                todo.push_back({nullptr, ' '});
                todo.push_back({n->kid[3], 0});
                break;
            case Kind::Apply:
                s << "(apply ";
                todo.push_back({nullptr, ')'});
                ops.push_back(op::INVALID);
                todo.push_back({n->kid[0], 0});
                todo.push_back({nullptr, ' '});
                todo.push_back({n->kid[1], 0});
                todo.push_back({nullptr, ' '});
                todo.push_back({n->kid[2], 0});
                break;
            case Kind::Invalid:
                s << "invalid";
                break;
        }
    }
}

}  // namespace lfb
