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
    // (same reason as libfive/src/tree/tree.cpp:27-69).
    std::vector<const Node*> todo{p};
    bool first = true;
    while (!todo.empty()) {
        const Node* n = todo.back();
        todo.pop_back();
        if (!first) {
            if (n->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) {
                continue;
            }
        }
        first = false;
        for (auto k : n->kid) {
            if (k) todo.push_back(k);
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
    n->serial = g_serial.fetch_add(1);
    n->refs.store(0);
    return Tree(n, true, false);
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
    if (op::arity(o) != 1) {
        return invalid();
    }
    if (a->kind == Kind::Constant) {
        return constant(fold_constant(o, a->value, 0.0f));
    }
    if (o == op::ABS) {
        if (a->kind == Kind::Unary &&
            (a->op == op::ABS || a->op == op::SQUARE)) {
            return a;
        }
    } else if (o == op::NEG) {
        if (a->kind == Kind::Unary && a->op == op::NEG) {
            return Tree(a->kid[0]);
        }
    }
    return make(Kind::Unary, o, 0, a.p, nullptr);
}

// Local simplifications follow tree.cpp:141-230, including the exact
// if / else-if chains (e.g. for ADD, a constant lhs stops the search even
// when it is non-zero).
Tree Tree::binary(int o, const Tree& a, const Tree& b)
{
    if (op::arity(o) != 2) {
        return invalid();
    }
    const bool ac = a->kind == Kind::Constant;
    const bool bc = b->kind == Kind::Constant;
    if (a.op() == op::CONSTANT && b.op() == op::CONSTANT) {
        return constant(fold_constant(o, a->value, b->value));
    }
    auto is_neg = [](const Tree& t) {
        return t->kind == Kind::Unary && t->op == op::NEG;
    };
    if (o == op::DIV) {
        if (bc && b->value == 1.0f) {
            return a;
        }
    } else if (o == op::ADD) {
        if (ac) {
            if (a->value == 0.0f) return b;
        } else if (bc) {
            if (b->value == 0.0f) return a;
        } else if (a->kind == Kind::Unary) {
            if (a->op == op::NEG) return b - Tree(a->kid[0]);
        } else if (b->kind == Kind::Unary) {
            if (b->op == op::NEG) return a - Tree(b->kid[0]);
        }
    } else if (o == op::SUB) {
        if (ac) {
            if (a->value == 0.0f) return -b;
        } else if (bc) {
            if (b->value == 0.0f) return a;
        } else if (is_neg(b)) {
            return a + Tree(b->kid[0]);
        }
    } else if (o == op::MUL) {
        if (ac) {
            if (a->value == 0) return a;
            if (a->value == 1) return b;
            if (a->value == -1) return -b;
        } else if (bc) {
            if (b->value == 0) return b;
            if (b->value == 1) return a;
            if (b->value == -1) return -a;
        } else if (a.p == b.p) {
            return unary(op::SQUARE, a);
        }
    } else if (o == op::NTH_ROOT || o == op::POW) {
        if (bc && b->value == 1.0f) {
            return a;
        }
    } else if (o == op::MIN || o == op::MAX) {
        if (a.p == b.p) {
            return a;
        }
    }
    return make(Kind::Binary, o, 0, a.p, b.p);
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
    std::unordered_map<const Node*, unsigned> count;
    std::vector<const Node*> todo{p};
    auto nkids = [](const Node* n) {
        return n->kind == Kind::Unary ? 1 : n->kind == Kind::Binary ? 2 : 0;
    };
    while (!todo.empty()) {
        const Node* n = todo.back();
        todo.pop_back();
        for (int i = 0; i < nkids(n); ++i) {
            if (count[n->kid[i]]++ == 0) {
                todo.push_back(n->kid[i]);
            }
        }
    }
    std::vector<const Node*> flat;
    todo.push_back(p);
    while (!todo.empty()) {
        const Node* n = todo.back();
        todo.pop_back();
        flat.push_back(n);
        for (int i = 0; i < nkids(n); ++i) {
            if (--count.at(n->kid[i]) == 0) {
                todo.push_back(n->kid[i]);
            }
        }
    }
    std::reverse(flat.begin(), flat.end());
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

    std::unordered_map<Key, Tree, KeyHash> canonical;
    auto uniq = [&canonical](const Tree& t) -> Tree {
        const Key k = key_of(t.p);
        auto it = canonical.find(k);
        if (it != canonical.end()) {
            return it->second;
        }
        canonical.emplace(k, t);
        return t;
    };

    // Affine accumulators map a tree to its scale factor.  The iteration
    // order of this map does not matter: terms are sorted before use.
    struct AffineMap {
        std::unordered_map<const Node*, std::pair<Tree, float>> terms;
        void add(const Tree& t, float s)
        {
            auto it = terms.find(t.get());
            if (it == terms.end()) {
                terms.emplace(t.get(), std::make_pair(t, s));
            } else {
                it->second.second += s;
            }
        }
    };
    struct CommList {
        int op;
        std::vector<Tree> list;
    };

    std::vector<std::optional<AffineMap>> affine;
    affine.emplace_back(std::nullopt);
    std::vector<std::optional<CommList>> comm;
    comm.emplace_back(std::nullopt);

    struct Task {
        enum { DOWN, UP, UP_AFFINE, UP_COMM } type;
        const Node* t;
        float scale;
    };
    std::vector<Task> todo{{Task::DOWN, p, 1.0f}};
    std::vector<Tree> out;

    auto deliver = [&](const Tree& self, float scale) {
        if (affine.back().has_value()) {
            if (self->kind == Kind::Constant) {
                affine.back()->add(one(), scale * self->value);
            } else {
                affine.back()->add(self, scale);
            }
        } else if (comm.back().has_value()) {
            comm.back()->list.push_back(self);
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
            comm.emplace_back(std::nullopt);
            affine.emplace_back(std::nullopt);

            bool marked_affine = false;
            auto mark_affine = [&]() {
                todo.pop_back();
                affine.pop_back();
                if (!affine.back().has_value()) {
                    affine.emplace_back(AffineMap());
                    todo.push_back({Task::UP_AFFINE, nullptr, 0.0f});
                } else {
                    comm.pop_back();
                }
                marked_affine = true;
            };
            auto mark_comm = [&](int o) {
                todo.pop_back();
                comm.pop_back();
                if (!comm.back().has_value() || comm.back()->op != o) {
                    comm.emplace_back(CommList{o, {}});
                    todo.push_back({Task::UP_COMM, nullptr, task.scale});
                } else {
                    affine.pop_back();
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
            affine.pop_back();
            comm.pop_back();
            const Node* d = task.t;
            Tree self = uniq(Tree(d));
            if (d->kind == Kind::Unary) {
                Tree a = std::move(out.back());
                out.pop_back();
                if (a.p != d->kid[0]) {
                    self = uniq(unary(d->op, a));
                }
            } else if (d->kind == Kind::Binary) {
                Tree a = std::move(out.back());
                out.pop_back();
                Tree b = std::move(out.back());
                out.pop_back();
                if (a.p != d->kid[0] || b.p != d->kid[1]) {
                    self = uniq(binary(d->op, a, b));
                }
            }
            deliver(self, task.scale);
        } else if (task.type == Task::UP_AFFINE) {
            AffineMap map = std::move(*affine.back());
            affine.pop_back();
            comm.pop_back();

            // Split into positive and negative terms; NaN scales go with the
            // positive terms and zero scales are dropped (tree.cpp:832-848).
            std::vector<std::pair<Tree, float>> pos, neg;
            for (auto& kv : map.terms) {
                const float s = kv.second.second;
                if (s > 0.0f) {
                    pos.push_back({kv.second.first, s});
                } else if (s < 0.0f) {
                    neg.push_back({kv.second.first, -s});
                } else if (s != 0.0f) {
                    pos.push_back({kv.second.first, s});
                }
            }
            auto order = [](const std::pair<Tree, float>& a,
                            const std::pair<Tree, float>& b) {
                if (a.second != b.second) {
                    return a.second < b.second;
                }
                return serial_less(a.first.get(), b.first.get());
            };
            std::sort(pos.begin(), pos.end(), order);
            std::sort(neg.begin(), neg.end(), order);

            auto collapse = [&](const std::vector<std::pair<Tree, float>>& v) {
                Tree acc = invalid();
                size_t i = 0;
                while (i < v.size()) {
                    const float mult = v[i].second;
                    Tree t = v[i].first;
                    ++i;
                    while (i < v.size() && v[i].second == mult) {
                        t = uniq(t + v[i].first);
                        ++i;
                    }
                    if (mult != 1) {
                        if (t == one()) {
                            t = uniq(constant(mult));
                        } else {
                            t = uniq(t * uniq(constant(mult)));
                        }
                    }
                    acc = acc.is_valid() ? uniq(acc + t) : t;
                }
                return acc.is_valid() ? acc : uniq(constant(0.0f));
            };
            const Tree P = collapse(pos);
            const Tree N = collapse(neg);
            Tree self = uniq(P - N);
            if (comm.back().has_value()) {
                comm.back()->list.push_back(self);
            } else {
                out.push_back(self);
            }
        } else {  // UP_COMM
            CommList c = std::move(*comm.back());
            comm.pop_back();
            affine.pop_back();
            std::sort(c.list.begin(), c.list.end(),
                      [](const Tree& a, const Tree& b) {
                          return serial_less(a.get(), b.get());
                      });
            auto end = c.list.end();
            if (op::is_idempotent(c.op)) {
                end = std::unique(c.list.begin(), c.list.end());
            }
            Tree self = c.list.front();
            for (auto it = c.list.begin() + 1; it != end; ++it) {
                self = uniq(binary(c.op, self, *it));
            }
            deliver(self, task.scale);
        }
    }
    return out.back().as_optimized();
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
