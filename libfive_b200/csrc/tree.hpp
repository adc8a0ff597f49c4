// Immutable, reference-counted expression DAG (the host side of the C API).
//
// This restates the behaviour of libfive::Tree
// (libfive/include/libfive/tree/tree.hpp:46-242, libfive/src/tree/tree.cpp):
//   * constructors apply the same local simplifications (tree.cpp:95-230),
//   * optimized() performs the same affine collapse / commutative-list
//     sorting / deduplication (tree.cpp:612-961),
//   * walk() gives the same leaves-to-root order (tree.cpp:530-594),
// because the clause order and slot numbering of the evaluation tape are a
// pure function of those three algorithms.  Where the reference orders
// nodes by heap address (sorting of commutative lists and affine terms),
// this implementation orders them by a creation serial number instead, which
// is one of the orders the reference can produce and is reproducible from
// run to run.
#pragma once
#include <atomic>
#include <cstdint>
#include <ostream>
#include <string>
#include <vector>

#include "opcode.hpp"

namespace lfb {

enum class Kind : uint8_t {
    Nullary, Unary, Binary, Constant, Remap, Apply, Invalid
};

struct Node {
    Kind kind;
    int op;
    uint32_t flags;
    uint64_t serial;
    float value;
    // Unary: kid[0]; Binary: kid[0], kid[1]
    // Remap: x, y, z, t; Apply: target, value, t
    const Node* kid[4];
    mutable std::atomic<uint32_t> refs;

    enum : uint32_t {
        HAS_REMAP = 1u << 0,
        HAS_XYZ = 1u << 2,
    };
};

class Tree {
public:
    Tree() : p(nullptr) {}
    ~Tree();
    Tree(const Tree& o) : p(o.p), optimized_flag(o.optimized_flag) { inc(); }
    Tree(Tree&& o) noexcept : p(o.p), optimized_flag(o.optimized_flag) { o.p = nullptr; }
    Tree& operator=(const Tree& o);
    Tree& operator=(Tree&& o) noexcept;

    /// Wraps a raw pointer handed out by release(), taking a new reference.
    explicit Tree(const Node* n) : p(n) { inc(); }
    /// Constant tree (value narrowed to float as in tree.cpp:71-75).
    static Tree constant(double v);

    static Tree X();
    static Tree Y();
    static Tree Z();
    static Tree var();
    static Tree invalid();

    static Tree nullary(int op);
    static Tree unary(int op, const Tree& a);
    static Tree binary(int op, const Tree& a, const Tree& b);

    Tree remap(const Tree& x, const Tree& y, const Tree& z) const;
    Tree apply(const Tree& var, const Tree& value) const;
    Tree flatten() const;
    Tree optimized() const;

    /// Leaves-to-root topological order of the (flattened) DAG.
    std::vector<const Node*> walk() const;
    /// The same order, and for the node at position i the positions of its
    /// operands in (*kid_pos)[2 i] and [2 i + 1] (UINT32_MAX where it has
    /// fewer), for passes that would otherwise look every operand up.  The
    /// tree must not need flattening (no remap / apply nodes).
    std::vector<const Node*> walk(std::vector<uint32_t>* kid_pos) const;
    size_t size() const;

    bool is_valid() const { return p && p->kind != Kind::Invalid; }
    const Node* get() const { return p; }
    const Node* operator->() const { return p; }
    int op() const;
    bool is_optimized() const { return optimized_flag; }

    /// Hands the pointer to a C caller without dropping the reference.
    const Node* release();
    /// Adopts a pointer from release() without taking a new reference.
    static Tree reclaim(const Node* n);

    bool operator==(const Tree& o) const { return p == o.p; }
    bool operator!=(const Tree& o) const { return p != o.p; }

    void print(std::ostream& s) const;

private:
    Tree(const Node* n, bool take_ref, bool opt) : p(n), optimized_flag(opt)
    {
        if (take_ref) inc();
    }
    static Tree make(Kind k, int op, float value, const Node* a,
                     const Node* b, const Node* c = nullptr,
                     const Node* d = nullptr);
    // unary() / binary() on borrowed node pointers, so that passes which
    // keep their operands alive elsewhere need no reference counting.
    static Tree unary_n(int op, const Node* a);
    static Tree binary_n(int op, const Node* a, const Node* b);
    static Tree one();
    Tree as_optimized() const { return Tree(p, true, true); }
    void inc() const
    {
        if (p) p->refs.fetch_add(1, std::memory_order_relaxed);
    }

    const Node* p;
    bool optimized_flag = false;
};

Tree operator+(const Tree& a, const Tree& b);
Tree operator-(const Tree& a, const Tree& b);
Tree operator*(const Tree& a, const Tree& b);
Tree operator/(const Tree& a, const Tree& b);
Tree operator-(const Tree& a);

/// Evaluates a single opcode on constant arguments (constant folding), using
/// the same float semantics as the point evaluators.
float fold_constant(int op, float a, float b);

}  // namespace lfb
