// Compile-time lowering of a rule AST (core/ast.hpp) into a bitwise network
// over 32-bit plane words.
//
// Representation.  A `word` holds one bit of 32 horizontally consecutive cells
// of one row (bit i = cell x0 + i, x0 a multiple of 32, least significant bit
// leftmost -- the order of the reference linear bit planes,
// include/memory/bit_planes_grid.hpp:255-263).  A value is `planes<B>`: B words,
// plane i holding bit i of the value of each of the 32 cells.  A condition is a
// single word.  Widths are tracked at compile time with exactly the rules of
// the reference bit-sliced integer (include/core/vector_int.hpp):
//   * from_constant<c> has width highest_bit(c) + 2, or 1 for c == 0 (:752-776)
//   * plus wraps at the wider operand's width (:227-286)
//   * modulo by 2^n truncates to n planes (bit_planes.hpp:163-182)
//   * comparisons zero-extend the narrower operand (:423-590)
//   * bit_and_ zero-fills and bit_or_ keeps the wider operand's extra planes (:625-700)
//   * if_then_else selects per cell with the condition mask (bit_planes.hpp:87-107)
// so every rule computes, cell for cell, what the reference standard evaluator
// computes (include/evaluators/standard.hpp).
//
// Neighbourhood access.  The engine hands the lowering three `row_feat`s (the
// rows above, at and below the output row) that it builds once per row when the
// row enters its rolling window: the row's planes shifted by dx = -1, 0, +1, and
// for every count target S of the rule the predicate "cell == S" at the three
// dx, with its full-adder (3 cells) and half-adder (2 cells) partial sums.  A
// Moore count is then a 3-operand carry-save addition of per-row partial sums
// (8 LOP3s) instead of the reference's chain of seven ripple adders.
//
// Only radius-1 neighbourhoods are supported (neighbor_at offsets in -1..1),
// the same limit as the reference tiled evaluator
// (include/evaluators/tiled_bit_planes.hpp:117, :202).
#ifndef CELLATO_B200_LOWER_CUH
#define CELLATO_B200_LOWER_CUH

#include <cstdint>
#include <type_traits>
#include <utility>

#include "../core/ast.hpp"

#if defined(__CUDACC__)
#define CB_HD __host__ __device__ __forceinline__
#else
#define CB_HD inline
#endif

namespace cellato::b200 {

using word = std::uint32_t;

constexpr int MAX_OUT_PLANES = 8;  // planes of a stored state

// ---------------------------------------------------------------- bit vectors
template <int B>
struct planes {
    static_assert(B >= 1, "a value has at least one plane");
    static constexpr int width = B;
    word p[B];
};

template <class T>
struct is_planes : std::false_type {};
template <int B>
struct is_planes<planes<B>> : std::true_type {};

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int cmin(int a, int b) { return a < b ? a : b; }

constexpr int highest_bit(long long v) {
    int h = -1;
    for (int i = 0; i < 62; ++i)
        if ((v >> i) & 1) h = i;
    return h;
}

// Width of a literal: highest set bit + 2 (one spare zero plane), 1 for zero.
constexpr int const_width(long long v) { return v == 0 ? 1 : highest_bit(v) + 2; }

constexpr int exact_log2(long long v) { return highest_bit(v); }

template <long long V>
CB_HD constexpr planes<const_width(V)> from_constant() {
    static_assert(V >= 0, "negative literals are not representable as bit planes");
    planes<const_width(V)> r;
#pragma unroll
    for (int i = 0; i < const_width(V); ++i) r.p[i] = ((V >> i) & 1) ? ~word(0) : word(0);
    return r;
}

// A condition used as a value is a one-plane vector.
CB_HD constexpr planes<1> as_planes(word w) { return planes<1>{{w}}; }
template <int B>
CB_HD constexpr planes<B> as_planes(planes<B> v) { return v; }

template <int N, int B>
CB_HD constexpr planes<N> resize(planes<B> a) {
    planes<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.p[i] = i < B ? a.p[i < B ? i : 0] : word(0);
    return r;
}

// Ripple-carry add modulo 2^max(A, B).
template <int A, int B>
CB_HD constexpr planes<cmax(A, B)> add(planes<A> a, planes<B> b) {
    constexpr int M = cmax(A, B), m = cmin(A, B);
    planes<M> r;
    word carry = 0;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i < m) {
            const word x = a.p[i] ^ b.p[i];
            r.p[i] = x ^ carry;
            carry = (a.p[i] & b.p[i]) | (carry & x);
        } else {
            const word w = A > B ? a.p[i < A ? i : 0] : b.p[i < B ? i : 0];
            r.p[i] = w ^ carry;
            carry = carry & w;
        }
    }
    return r;
}

template <int A, int B>
CB_HD constexpr planes<cmax(A, B)> bor(planes<A> a, planes<B> b) {
    constexpr int M = cmax(A, B);
    planes<M> r;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const word x = i < A ? a.p[i < A ? i : 0] : word(0);
        const word y = i < B ? b.p[i < B ? i : 0] : word(0);
        r.p[i] = x | y;
    }
    return r;
}

template <int A, int B>
CB_HD constexpr planes<cmax(A, B)> band(planes<A> a, planes<B> b) {
    constexpr int M = cmax(A, B);
    planes<M> r;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const word x = i < A ? a.p[i < A ? i : 0] : word(0);
        const word y = i < B ? b.p[i < B ? i : 0] : word(0);
        r.p[i] = x & y;
    }
    return r;
}

template <int B>
CB_HD constexpr planes<B> mask(planes<B> a, word m) {
#pragma unroll
    for (int i = 0; i < B; ++i) a.p[i] &= m;
    return a;
}

template <int A, int B>
CB_HD constexpr word eq(planes<A> a, planes<B> b) {
    word r = ~word(0);
#pragma unroll
    for (int i = 0; i < cmax(A, B); ++i) {
        const word x = i < A ? a.p[i < A ? i : 0] : word(0);
        const word y = i < B ? b.p[i < B ? i : 0] : word(0);
        r &= ~(x ^ y);
    }
    return r;
}

template <int A, int B>
CB_HD constexpr word ne(planes<A> a, planes<B> b) { return ~eq(a, b); }

// Unsigned a > b, most significant plane first.
template <int A, int B>
CB_HD constexpr word gt(planes<A> a, planes<B> b) {
    word result = 0, decided = 0;
#pragma unroll
    for (int i = cmax(A, B) - 1; i >= 0; --i) {
        const word x = i < A ? a.p[i < A ? i : 0] : word(0);
        const word y = i < B ? b.p[i < B ? i : 0] : word(0);
        result |= ~decided & x & ~y;
        decided |= x ^ y;
    }
    return result;
}

template <int A, int B>
CB_HD constexpr word lt(planes<A> a, planes<B> b) { return gt(b, a); }

// "all NB planes spell the constant S" -- equals_to<S> of a stored state.
template <int S, int NB>
CB_HD constexpr word eq_const(const word* p) {
    word r = ~word(0);
#pragma unroll
    for (int i = 0; i < NB; ++i) r &= ((S >> i) & 1) ? p[i] : ~p[i];
    return r;
}

// Full adder / half adder on words (each output is one LOP3).
CB_HD constexpr word xor3(word a, word b, word c) { return a ^ b ^ c; }
CB_HD constexpr word maj3(word a, word b, word c) { return (a & b) | (c & (a ^ b)); }

// Funnel shifts that bring a neighbour word's edge bit in.
// shl1(prev, cur): bit i = cur bit i-1, bit 0 = prev bit 31   (cell x-1)
// shr1(cur, next): bit i = cur bit i+1, bit 31 = next bit 0   (cell x+1)
CB_HD word shl1(word prev, word cur) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_l(prev, cur, 1);
#else
    return (cur << 1) | (prev >> 31);
#endif
}
CB_HD word shr1(word cur, word next) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_r(cur, next, 1);
#else
    return (cur >> 1) | (next << 31);
#endif
}

// ------------------------------------------------------- collecting targets
// Dictionary indices S of every count_neighbors<state_constant<V>, ...> node.
template <int... S>
struct ilist {
    static constexpr int size = sizeof...(S);
};

template <class A, class B>
struct icat;
template <int... A, int... B>
struct icat<ilist<A...>, ilist<B...>> {
    using type = ilist<A..., B...>;
};

template <class... Ls>
struct icat_all {
    using type = ilist<>;
};
template <class L, class... Ls>
struct icat_all<L, Ls...> {
    using type = typename icat<L, typename icat_all<Ls...>::type>::type;
};

template <class L, int S>
struct icontains;
template <int S, int... Xs>
struct icontains<ilist<Xs...>, S> {
    static constexpr bool value = ((Xs == S) || ...);
};

template <class L>
struct idedup {
    using type = ilist<>;
};
template <int X, int... Xs>
struct idedup<ilist<X, Xs...>> {
    using rest = typename idedup<ilist<Xs...>>::type;
    using type = std::conditional_t<icontains<rest, X>::value, rest, typename icat<ilist<X>, rest>::type>;
};

template <class L, int S>
struct iindex;
template <int S, int X, int... Xs>
struct iindex<ilist<X, Xs...>, S> {
    static constexpr int value = (X == S) ? 0 : 1 + iindex<ilist<Xs...>, S>::value;
};
template <int S>
struct iindex<ilist<>, S> {
    static constexpr int value = 0;
};

namespace ast = cellato::ast;

template <class Dict, class E>
struct count_targets {
    using type = ilist<>;
};

template <class Dict, class N>
struct count_targets_nb {
    using type = ilist<>;
};

template <class Dict, auto V, class N>
struct count_targets<Dict, ast::count_neighbors<ast::state_constant<V>, N>> {
    using type = ilist<Dict::state_to_index(V)>;
};
template <class Dict, class T, class N>
struct count_targets<Dict, ast::count_neighbors<T, N>> {
    using type = typename count_targets<Dict, T>::type;
};
template <class Dict, class C, class T, class E>
struct count_targets<Dict, ast::if_then_else<C, T, E>> {
    using type = typename icat_all<typename count_targets<Dict, C>::type, typename count_targets<Dict, T>::type,
                                   typename count_targets<Dict, E>::type>::type;
};
template <class Dict, class V>
struct count_targets<Dict, ast::not_<V>> {
    using type = typename count_targets<Dict, V>::type;
};
template <class Dict, class V, int b>
struct count_targets<Dict, ast::has_bit_set<V, b>> {
    using type = typename count_targets<Dict, V>::type;
};
template <class Dict, class... As>
struct count_targets<Dict, ast::alternate_algorithms<As...>> {
    using type = typename icat_all<typename count_targets<Dict, As>::type...>::type;
};
#define CB_BINARY_TARGETS(NODE)                                                                             \
    template <class Dict, class L, class R>                                                                 \
    struct count_targets<Dict, ast::NODE<L, R>> {                                                           \
        using type =                                                                                        \
            typename icat<typename count_targets<Dict, L>::type, typename count_targets<Dict, R>::type>::type; \
    };
CB_BINARY_TARGETS(and_)
CB_BINARY_TARGETS(or_)
CB_BINARY_TARGETS(bit_and_)
CB_BINARY_TARGETS(bit_or_)
CB_BINARY_TARGETS(plus)
CB_BINARY_TARGETS(modulo)
CB_BINARY_TARGETS(equals)
CB_BINARY_TARGETS(not_equals)
CB_BINARY_TARGETS(greater_than)
CB_BINARY_TARGETS(less_than)
#undef CB_BINARY_TARGETS

template <class Dict, class E>
using targets_of = typename idedup<typename count_targets<Dict, E>::type>::type;

// ------------------------------------------------- which features a rule reads
// uses_shift<E>: E reads neighbour planes at dx != 0 (the row's planes shifted
// by one cell); uses_sums<E>: E reads full Moore / von Neumann counts of a fixed
// state (the per-row partial sums).  Only these features are computed.
template <class E>
struct is_state_const : std::false_type {};
template <auto V>
struct is_state_const<ast::state_constant<V>> : std::true_type {};

template <class E>
struct is_count : std::false_type {};
template <class T, class N>
struct is_count<ast::count_neighbors<T, N>> : std::true_type {};

template <class E>
struct is_count_test : std::false_type {};  // greater_than<count_neighbors<T, moore | von Neumann>, constant<Z>>
template <class T, auto Z>
struct is_count_test<ast::greater_than<ast::count_neighbors<T, ast::moore_8_neighbors>, ast::constant<Z>>>
    : std::true_type {};
template <class T, auto Z>
struct is_count_test<ast::greater_than<ast::count_neighbors<T, ast::von_neumann_4_neighbors>, ast::constant<Z>>>
    : std::true_type {};

template <class E, class = void>
struct uses_shift : std::false_type {};
template <class E, class = void>
struct uses_sums : std::false_type {};

template <int dx, int dy>
struct uses_shift<ast::neighbor_at<dx, dy>, void> : std::bool_constant<dx != 0> {};
template <>
struct uses_shift<ast::margolus_180_neighbor, void> : std::true_type {};
template <class T, class N>
struct uses_shift<ast::count_neighbors<T, N>, void> : std::bool_constant<!is_state_const<T>::value> {};
template <class V, int b>
struct uses_shift<ast::has_bit_set<V, b>, void> : uses_shift<V> {};
template <template <class...> class N, class... Ch>
struct uses_shift<N<Ch...>, std::enable_if_t<!is_count<N<Ch...>>::value>>
    : std::bool_constant<(uses_shift<Ch>::value || ...)> {};

template <class T, class N>
struct uses_sums<ast::count_neighbors<T, N>, void>
    : std::bool_constant<(is_state_const<T>::value && (std::is_same_v<N, ast::moore_8_neighbors> ||
                                                        std::is_same_v<N, ast::von_neumann_4_neighbors>)) ||
                         uses_sums<T>::value> {};
template <class V, int b>
struct uses_sums<ast::has_bit_set<V, b>, void> : uses_sums<V> {};
template <template <class...> class N, class... Ch>
struct uses_sums<N<Ch...>, std::enable_if_t<!is_count<N<Ch...>>::value && !is_count_test<N<Ch...>>::value>>
    : std::bool_constant<(uses_sums<Ch>::value || ...)> {};
// "count > 0" reads the predicates only (the OR fast path below)
template <class T, auto Z>
struct uses_sums<ast::greater_than<ast::count_neighbors<T, ast::moore_8_neighbors>, ast::constant<Z>>, void>
    : std::bool_constant<Z != 0 || uses_sums<T>::value> {};
template <class T, auto Z>
struct uses_sums<ast::greater_than<ast::count_neighbors<T, ast::von_neumann_4_neighbors>, ast::constant<Z>>, void>
    : std::bool_constant<Z != 0 || uses_sums<T>::value> {};

// uses_any<E>: E tests "any Moore neighbour is S" (count > 0) for a fixed S,
// which reads the per-row ORs of the predicates.
template <class E, class = void>
struct uses_any : std::false_type {};
template <class V, int b>
struct uses_any<ast::has_bit_set<V, b>, void> : uses_any<V> {};
template <template <class...> class N, class... Ch>
struct uses_any<N<Ch...>, std::enable_if_t<!is_count_test<N<Ch...>>::value>>
    : std::bool_constant<(uses_any<Ch>::value || ...)> {};
template <class T, auto Z>
struct uses_any<ast::greater_than<ast::count_neighbors<T, ast::moore_8_neighbors>, ast::constant<Z>>, void>
    : std::bool_constant<(Z == 0 && is_state_const<T>::value) || uses_any<T>::value> {};
template <class T, auto Z>
struct uses_any<ast::greater_than<ast::count_neighbors<T, ast::von_neumann_4_neighbors>, ast::constant<Z>>, void>
    : uses_any<T> {};

// ------------------------------------------------------------ per-row cache
// Predicate "cell == S" at dx = -1, 0, +1 and its partial sums.
struct count_cache {
    word P[3];   // P[dx + 1]
    word o2, o3; // P[0] | P[2], P[0] | P[1] | P[2]  (any-neighbour tests)
    word s3, c3; // P[0] + P[1] + P[2]  (sum, carry)
    word s2, c2; // P[0] + P[2]
};

template <int NB, class Targets>
struct row_feat {
    word sh[3][NB];  // sh[dx + 1][plane]
    count_cache cc[Targets::size > 0 ? Targets::size : 1];
};

// Predicates "cell == S" of one word for every count target S.
template <class Targets>
struct pred_set {
    word p[Targets::size > 0 ? Targets::size : 1];
};

template <int NB, int... S>
CB_HD pred_set<ilist<S...>> preds_of_impl(const word* C, ilist<S...>) {
    pred_set<ilist<S...>> r{};
    int k = 0;
    ((r.p[k++] = eq_const<S, NB>(C)), ...);
    (void)k;
    return r;
}

// Builds a row's features for one word from its own planes (C), the words to
// its left and right (L, R: only bit 31 / bit 0 matter, read only when SHIFT)
// and the count-target predicates of the three words.
template <int NB, class Targets, bool SHIFT, bool SUMS, bool ANY = false>
CB_HD row_feat<NB, Targets> make_row_feat(const word* C, const word* L, const word* R, const pred_set<Targets>& pc,
                                          const pred_set<Targets>& pl, const pred_set<Targets>& pr) {
    row_feat<NB, Targets> f;
#pragma unroll
    for (int p = 0; p < NB; ++p) {
        f.sh[1][p] = C[p];
        if constexpr (SHIFT) {
            f.sh[0][p] = shl1(L[p], C[p]);
            f.sh[2][p] = shr1(C[p], R[p]);
        }
    }
#pragma unroll
    for (int k = 0; k < Targets::size; ++k) {
        count_cache& c = f.cc[k];
        c.P[0] = shl1(pl.p[k], pc.p[k]);  // predicate first, shift second
        c.P[1] = pc.p[k];
        c.P[2] = shr1(pc.p[k], pr.p[k]);
        if constexpr (SUMS) {
            c.s3 = xor3(c.P[0], c.P[1], c.P[2]);
            c.c3 = maj3(c.P[0], c.P[1], c.P[2]);
            c.s2 = c.P[0] ^ c.P[2];
            c.c2 = c.P[0] & c.P[2];
        }
        if constexpr (ANY) {
            c.o2 = c.P[0] | c.P[2];
            c.o3 = c.o2 | c.P[1];
        }
    }
    return f;
}

// Evaluation context of one output word.  TP is the parity of the time step
// (a compile-time constant: the engines instantiate both), ypar the parity of
// the output row's global y.
template <class RF, int TP>
struct ctx {
    static constexpr int tp = TP;
    static constexpr bool symbolic = false;
    const RF& up;
    const RF& mid;
    const RF& dn;
    int ypar;

    template <int dy>
    CB_HD constexpr const RF& row() const {
        if constexpr (dy < 0)
            return up;
        else if constexpr (dy > 0)
            return dn;
        else
            return mid;
    }
    // The vertical Margolus partner of the output row is y+1 when (y + t) is
    // even and y-1 otherwise (include/evaluators/standard.hpp:183-197).  The
    // choice is made per word value (a select), never by picking a struct.
    CB_HD constexpr bool margolus_down() const { return ((ypar ^ TP) == 0); }
    CB_HD constexpr word pick(word down_value, word up_value) const { return margolus_down() ? down_value : up_value; }
};

// Bits whose horizontal Margolus partner is x+1: even x on even steps, odd x
// on odd steps.  Word origins are multiples of 32, so x parity = bit parity.
template <int TP>
CB_HD constexpr word margolus_right_mask() { return TP == 0 ? word(0x55555555u) : word(0xAAAAAAAAu); }

// --------------------------------------------------------------- the nodes
template <class Dict, class Targets, class E>
struct lower {
    static_assert(sizeof(E) == 0, "AST node not supported by the B200 lowering");
};

// Signal nodes: the leaves of a rule's state-transition logic -- neighbour
// states, neighbourhood counts and "any neighbour is ..." tests.  Everything
// above them is a pure per-cell boolean function (see rule_net below).
template <class E>
struct is_signal : std::false_type {};
template <int dx, int dy>
struct is_signal<ast::neighbor_at<dx, dy>> : std::true_type {};
template <class T, class N>
struct is_signal<ast::count_neighbors<T, N>> : std::true_type {};
template <>
struct is_signal<ast::margolus_180_neighbor> : std::true_type {};
template <class T, auto Z>
struct is_signal<ast::greater_than<ast::count_neighbors<T, ast::moore_8_neighbors>, ast::constant<Z>>>
    : std::bool_constant<Z == 0> {};
template <class T, auto Z>
struct is_signal<ast::greater_than<ast::count_neighbors<T, ast::von_neumann_4_neighbors>, ast::constant<Z>>>
    : std::bool_constant<Z == 0> {};

// Evaluate node E (free function, so that node bodies can recurse by name).
// In a symbolic context (compile-time truth-table evaluation) signal nodes
// yield the truth-table patterns of their input variables.
template <class Dict, class Targets, class E, class C>
CB_HD constexpr auto ev(const C& c) {
    if constexpr (C::symbolic && is_signal<E>::value)
        return c.template sig<E>();
    else
        return lower<Dict, Targets, E>::eval(c);
}

template <class T>
CB_HD constexpr word as_cond(T v) {
    if constexpr (std::is_same_v<T, word>)
        return v;
    else {
        static_assert(std::is_same_v<T, planes<1>>, "a condition must be a single plane");
        return v.p[0];
    }
}

template <class Dict, class Targets, auto V>
struct lower<Dict, Targets, ast::constant<V>> {
    template <class C>
    CB_HD static constexpr auto eval(const C&) { return from_constant<(long long)V>(); }
};

template <class Dict, class Targets, auto V>
struct lower<Dict, Targets, ast::state_constant<V>> {
    template <class C>
    CB_HD static constexpr auto eval(const C&) { return from_constant<(long long)Dict::state_to_index(V)>(); }
};

template <class Dict, class Targets, int dx, int dy>
struct lower<Dict, Targets, ast::neighbor_at<dx, dy>> {
    static_assert(dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1, "neighbor_at offsets are limited to -1..1");
    static constexpr int NB = Dict::needed_bits;
    template <class C>
    CB_HD static constexpr planes<NB> eval(const C& c) {
        planes<NB> r;
        const auto& row = c.template row<dy>();
#pragma unroll
        for (int p = 0; p < NB; ++p) r.p[p] = row.sh[dx + 1][p];
        return r;
    }
};

template <class Dict, class Targets, class Cn, class T, class E>
struct lower<Dict, Targets, ast::if_then_else<Cn, T, E>> {
    template <class C>
    CB_HD static constexpr auto eval(const C& c) {
        const word m = as_cond(ev<Dict, Targets, Cn>(c));
        auto t = ev<Dict, Targets, T>(c);
        auto e = ev<Dict, Targets, E>(c);
        if constexpr (std::is_same_v<decltype(t), word> && std::is_same_v<decltype(e), word>)
            return word((t & m) | (e & ~m));
        else
            return bor(mask(as_planes(t), m), mask(as_planes(e), ~m));
    }
};

template <class Dict, class Targets, class L, class R>
struct lower<Dict, Targets, ast::and_<L, R>> {
    template <class C>
    CB_HD static constexpr word eval(const C& c) {
        return as_cond(ev<Dict, Targets, L>(c)) & as_cond(ev<Dict, Targets, R>(c));
    }
};

template <class Dict, class Targets, class L, class R>
struct lower<Dict, Targets, ast::or_<L, R>> {
    template <class C>
    CB_HD static constexpr word eval(const C& c) {
        return as_cond(ev<Dict, Targets, L>(c)) | as_cond(ev<Dict, Targets, R>(c));
    }
};

template <class Dict, class Targets, class V>
struct lower<Dict, Targets, ast::not_<V>> {
    template <class C>
    CB_HD static constexpr word eval(const C& c) { return ~as_cond(ev<Dict, Targets, V>(c)); }
};

template <class Dict, class Targets, class L, class R>
struct lower<Dict, Targets, ast::bit_and_<L, R>> {
    template <class C>
    CB_HD static constexpr auto eval(const C& c) {
        auto a = ev<Dict, Targets, L>(c);
        auto b = ev<Dict, Targets, R>(c);
        if constexpr (std::is_same_v<decltype(a), word> && std::is_same_v<decltype(b), word>)
            return word(a & b);
        else
            return band(as_planes(a), as_planes(b));
    }
};

template <class Dict, class Targets, class L, class R>
struct lower<Dict, Targets, ast::bit_or_<L, R>> {
    template <class C>
    CB_HD static constexpr auto eval(const C& c) {
        auto a = ev<Dict, Targets, L>(c);
        auto b = ev<Dict, Targets, R>(c);
        if constexpr (std::is_same_v<decltype(a), word> && std::is_same_v<decltype(b), word>)
            return word(a | b);
        else
            return bor(as_planes(a), as_planes(b));
    }
};

template <class Dict, class Targets, class L, class R>
struct lower<Dict, Targets, ast::plus<L, R>> {
    template <class C>
    CB_HD static constexpr auto eval(const C& c) {
        return add(as_planes(ev<Dict, Targets, L>(c)), as_planes(ev<Dict, Targets, R>(c)));
    }
};

template <class Dict, class Targets, class L, auto V>
struct lower<Dict, Targets, ast::modulo<L, ast::constant<V>>> {
    static_assert(V > 0 && (V & (V - 1)) == 0, "only modulo by a power of two is supported");
    template <class C>
    CB_HD static constexpr auto eval(const C& c) {
        return resize<exact_log2(V)>(as_planes(ev<Dict, Targets, L>(c)));
    }
};

#define CB_COMPARE(NODE, FN)                                                              \
    template <class Dict, class Targets, class L, class R>                                \
    struct lower<Dict, Targets, ast::NODE<L, R>> {                                        \
        template <class C>                                                                \
        CB_HD static constexpr word eval(const C& c) {                                              \
            return FN(as_planes(ev<Dict, Targets, L>(c)), as_planes(ev<Dict, Targets, R>(c))); \
        }                                                                                 \
    };
CB_COMPARE(equals, eq)
CB_COMPARE(not_equals, ne)
CB_COMPARE(greater_than, gt)
CB_COMPARE(less_than, lt)
#undef CB_COMPARE

template <class Dict, class Targets, class V, int b>
struct lower<Dict, Targets, ast::has_bit_set<V, b>> {
    template <class C>
    CB_HD static constexpr word eval(const C& c) {
        auto v = as_planes(ev<Dict, Targets, V>(c));
        static_assert(b >= 0 && b < decltype(v)::width, "has_bit_set bit beyond the value's width");
        return v.p[b];
    }
};

template <class Dict, class Targets, class Even, class Odd>
struct lower<Dict, Targets, ast::alternate_algorithms<Even, Odd>> {
    template <class C>
    CB_HD static constexpr auto eval(const C& c) {
        if constexpr (C::tp == 0)
            return ev<Dict, Targets, Even>(c);
        else
            return ev<Dict, Targets, Odd>(c);
    }
};

// Moore count of a fixed state: rows above and below contribute their 3-cell
// sums, the own row its 2-cell sum; a 3-operand carry-save add gives 4 planes.
template <class Dict, class Targets, auto V>
struct lower<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::moore_8_neighbors>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class C>
    CB_HD static constexpr planes<4> eval(const C& c) {
        const count_cache& a = c.up.cc[slot];
        const count_cache& b = c.dn.cc[slot];
        const count_cache& m = c.mid.cc[slot];
        const word s0 = xor3(a.s3, b.s3, m.s2);
        const word k1 = maj3(a.s3, b.s3, m.s2);
        const word t1 = xor3(a.c3, b.c3, m.c2);
        const word t2 = maj3(a.c3, b.c3, m.c2);
        const word s1 = k1 ^ t1;
        const word k2 = k1 & t1;
        return planes<4>{{s0, s1, t2 ^ k2, t2 & k2}};
    }
};

// von Neumann count of a fixed state: cells above and below plus the own row's
// left+right sum; 3 planes.
template <class Dict, class Targets, auto V>
struct lower<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::von_neumann_4_neighbors>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class C>
    CB_HD static constexpr planes<3> eval(const C& c) {
        const word u = c.up.cc[slot].P[1], d = c.dn.cc[slot].P[1];
        const count_cache& m = c.mid.cc[slot];
        const word s0 = xor3(u, d, m.s2);
        const word k1 = maj3(u, d, m.s2);
        return planes<3>{{s0, m.c2 ^ k1, m.c2 & k1}};
    }
};

// "any neighbour is S": a plain OR of the predicates (the count > 0 fast path
// of include/evaluators/bit_planes.hpp:598-628, and its von Neumann analogue).
template <class Dict, class Targets, auto V, auto Z>
struct lower<Dict, Targets,
             ast::greater_than<ast::count_neighbors<ast::state_constant<V>, ast::moore_8_neighbors>, ast::constant<Z>>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class C>
    CB_HD static constexpr word eval(const C& c) {
        if constexpr (Z == 0) {
            // the rows above and below contribute their 3-cell ORs, the own
            // row its 2-cell OR (row features built with uses_any)
            return c.up.cc[slot].o3 | c.dn.cc[slot].o3 | c.mid.cc[slot].o2;
        } else {
            // through ev, so that a symbolic context substitutes the count signal
            return gt(ev<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::moore_8_neighbors>>(c),
                      from_constant<(long long)Z>());
        }
    }
};

template <class Dict, class Targets, auto V, auto Z>
struct lower<Dict, Targets,
             ast::greater_than<ast::count_neighbors<ast::state_constant<V>, ast::von_neumann_4_neighbors>,
                               ast::constant<Z>>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class C>
    CB_HD static constexpr word eval(const C& c) {
        if constexpr (Z == 0) {
            return c.up.cc[slot].P[1] | c.dn.cc[slot].P[1] | c.mid.cc[slot].P[0] | c.mid.cc[slot].P[2];
        } else {
            return gt(ev<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::von_neumann_4_neighbors>>(c),
                      from_constant<(long long)Z>());
        }
    }
};

// Counts against a target that depends on the cell itself (e.g. cyclic's
// (state + 1) mod 32): compare each neighbour's planes with the target.
template <int NB, class T, class RF>
CB_HD constexpr word neighbour_eq(const RF& row, int dxi, const T& target) {
    planes<NB> n;
#pragma unroll
    for (int p = 0; p < NB; ++p) n.p[p] = row.sh[dxi][p];
    return eq(n, target);
}

template <int N>
CB_HD constexpr planes<4> popcount8(const word (&x)[N]) {
    static_assert(N == 8);
    // carry-save tree: 4 full adders + 3 half adders
    const word a0 = xor3(x[0], x[1], x[2]), a1 = maj3(x[0], x[1], x[2]);
    const word b0 = xor3(x[3], x[4], x[5]), b1 = maj3(x[3], x[4], x[5]);
    const word c0 = xor3(x[6], x[7], a0), c1 = maj3(x[6], x[7], a0);
    const word s0 = b0 ^ c0, d1 = b0 & c0;
    const word e1 = xor3(a1, b1, c1), e2 = maj3(a1, b1, c1);
    const word s1 = e1 ^ d1, f2 = e1 & d1;
    return planes<4>{{s0, s1, e2 ^ f2, e2 & f2}};
}

template <class Dict, class Targets, class T>
struct lower<Dict, Targets, ast::count_neighbors<T, ast::moore_8_neighbors>> {
    static constexpr int NB = Dict::needed_bits;
    template <class C>
    CB_HD static constexpr planes<4> eval(const C& c) {
        const auto t = as_planes(ev<Dict, Targets, T>(c));
        const word x[8] = {neighbour_eq<NB>(c.up, 0, t),  neighbour_eq<NB>(c.up, 1, t),
                           neighbour_eq<NB>(c.up, 2, t),  neighbour_eq<NB>(c.mid, 0, t),
                           neighbour_eq<NB>(c.mid, 2, t), neighbour_eq<NB>(c.dn, 0, t),
                           neighbour_eq<NB>(c.dn, 1, t),  neighbour_eq<NB>(c.dn, 2, t)};
        return popcount8(x);
    }
};

template <class Dict, class Targets, class T>
struct lower<Dict, Targets, ast::count_neighbors<T, ast::von_neumann_4_neighbors>> {
    static constexpr int NB = Dict::needed_bits;
    template <class C>
    CB_HD static constexpr planes<3> eval(const C& c) {
        const auto t = as_planes(ev<Dict, Targets, T>(c));
        const word u = neighbour_eq<NB>(c.up, 1, t), d = neighbour_eq<NB>(c.dn, 1, t);
        const word l = neighbour_eq<NB>(c.mid, 0, t), r = neighbour_eq<NB>(c.mid, 2, t);
        const word s0 = xor3(u, d, l), k1 = maj3(u, d, l);
        const word s0b = s0 ^ r, k1b = s0 & r;
        return planes<3>{{s0b, k1 ^ k1b, k1 & k1b}};
    }
};

template <class Dict, class Targets, class T, auto Z>
struct lower<Dict, Targets, ast::greater_than<ast::count_neighbors<T, ast::moore_8_neighbors>, ast::constant<Z>>> {
    static constexpr int NB = Dict::needed_bits;
    template <class C>
    CB_HD static constexpr word eval(const C& c) {
        if constexpr (Z == 0) {
            const auto t = as_planes(ev<Dict, Targets, T>(c));
            return neighbour_eq<NB>(c.up, 0, t) | neighbour_eq<NB>(c.up, 1, t) | neighbour_eq<NB>(c.up, 2, t) |
                   neighbour_eq<NB>(c.mid, 0, t) | neighbour_eq<NB>(c.mid, 2, t) | neighbour_eq<NB>(c.dn, 0, t) |
                   neighbour_eq<NB>(c.dn, 1, t) | neighbour_eq<NB>(c.dn, 2, t);
        } else {
            return gt(lower<Dict, Targets, ast::count_neighbors<T, ast::moore_8_neighbors>>::eval(c),
                      from_constant<(long long)Z>());
        }
    }
};

// Margolus 2x2 block count of a fixed state (standard.hpp:175-205): the block
// of a cell is itself, its horizontal partner, its vertical partner and the
// diagonal one.  Per row, pair = P(x) + P(partner x); count = pair(own row) +
// pair(partner row).
template <class Dict, class Targets, auto V>
struct lower<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::margolus_alternating_neighborhood>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class RF, int TP>
    CB_HD static constexpr planes<3> eval(const ctx<RF, TP>& c) {
        constexpr word M = margolus_right_mask<TP>();
        const count_cache& m = c.mid.cc[slot];
        const count_cache& u = c.up.cc[slot];
        const count_cache& d = c.dn.cc[slot];
        const word v0 = c.pick(d.P[0], u.P[0]), v1 = c.pick(d.P[1], u.P[1]), v2 = c.pick(d.P[2], u.P[2]);
        const word hm = (m.P[2] & M) | (m.P[0] & ~M);
        const word hv = (v2 & M) | (v0 & ~M);
        const word a0 = m.P[1] ^ hm, a1 = m.P[1] & hm;
        const word b0 = v1 ^ hv, b1 = v1 & hv;
        const word k = a0 & b0;
        return planes<3>{{a0 ^ b0, xor3(a1, b1, k), maj3(a1, b1, k)}};
    }
};

// State of the diagonally opposite cell of the block (standard.hpp:207-241).
template <class Dict, class Targets>
struct lower<Dict, Targets, ast::margolus_180_neighbor> {
    static constexpr int NB = Dict::needed_bits;
    template <class RF, int TP>
    CB_HD static constexpr planes<NB> eval(const ctx<RF, TP>& c) {
        constexpr word M = margolus_right_mask<TP>();
        planes<NB> r;
#pragma unroll
        for (int p = 0; p < NB; ++p) {
            const word right = c.pick(c.dn.sh[2][p], c.up.sh[2][p]);
            const word left = c.pick(c.dn.sh[0][p], c.up.sh[0][p]);
            r.p[p] = (right & M) | (left & ~M);
        }
        return r;
    }
};

// ------------------------------------------------ LOP3 network synthesis
// A rule is a per-cell boolean function of its signals.  When the signals of a
// rule add up to at most 6 input bits, the output planes are synthesised at
// compile time into a minimal-ish LOP3 network: the rule is evaluated once,
// symbolically, on truth-table patterns (bit m of variable j's pattern = bit j
// of m), and each output truth table is decomposed by Shannon expansion down to
// sub-functions of at most three variables, each one LOP3.  Sub-functions are
// shared across outputs by truth table.

template <class... Ts>
struct tlist {
    static constexpr int size = sizeof...(Ts);
};

template <class L, class T>
struct tl_has;
template <class T, class... Ts>
struct tl_has<tlist<Ts...>, T> : std::bool_constant<(std::is_same_v<T, Ts> || ...)> {};

template <class L, class T>
struct tl_add {
    using type = std::conditional_t<tl_has<L, T>::value, L, L>;
};
template <class T, class... Ts>
struct tl_add<tlist<Ts...>, T> {
    using type = std::conditional_t<tl_has<tlist<Ts...>, T>::value, tlist<Ts...>, tlist<Ts..., T>>;
};

template <class L, class R>
struct tl_merge;
template <class L>
struct tl_merge<L, tlist<>> {
    using type = L;
};
template <class L, class T, class... Ts>
struct tl_merge<L, tlist<T, Ts...>> {
    using type = typename tl_merge<typename tl_add<L, T>::type, tlist<Ts...>>::type;
};

// signals_of<E, TP>: the signal nodes E depends on (alternate_algorithms
// contributes only the branch of step parity TP).
template <class E, int TP, class = void>
struct signals_of {
    using type = tlist<>;
};
template <class E, int TP>
struct signals_of<E, TP, std::enable_if_t<is_signal<E>::value>> {
    using type = tlist<E>;
};
template <class E>
struct is_alternation : std::false_type {};
template <class... As>
struct is_alternation<ast::alternate_algorithms<As...>> : std::true_type {};

template <template <class...> class N, class... Ch, int TP>
struct signals_of<N<Ch...>, TP, std::enable_if_t<!is_signal<N<Ch...>>::value && !is_alternation<N<Ch...>>::value>> {
    template <class Acc, class... Rest>
    struct fold {
        using type = Acc;
    };
    template <class Acc, class X, class... Rest>
    struct fold<Acc, X, Rest...> {
        using type = typename fold<typename tl_merge<Acc, typename signals_of<X, TP>::type>::type, Rest...>::type;
    };
    using type = typename fold<tlist<>, Ch...>::type;
};
template <class Even, class Odd, int TP>
struct signals_of<ast::alternate_algorithms<Even, Odd>, TP, void> {
    using type = typename signals_of<std::conditional_t<TP == 0, Even, Odd>, TP>::type;
};
template <class V, int b, int TP>
struct signals_of<ast::has_bit_set<V, b>, TP, void> {
    using type = typename signals_of<V, TP>::type;
};

// Number of planes a signal contributes.
template <class Dict, class S>
struct signal_width {
    static constexpr int value = Dict::needed_bits;  // neighbor_at, margolus_180_neighbor
};
template <class Dict, class T>
struct signal_width<Dict, ast::count_neighbors<T, ast::moore_8_neighbors>> {
    static constexpr int value = 4;
};
template <class Dict, class T>
struct signal_width<Dict, ast::count_neighbors<T, ast::von_neumann_4_neighbors>> {
    static constexpr int value = 3;
};
template <class Dict, class T>
struct signal_width<Dict, ast::count_neighbors<T, ast::margolus_alternating_neighborhood>> {
    static constexpr int value = 3;
};
template <class Dict, class T, auto Z>
struct signal_width<Dict, ast::greater_than<ast::count_neighbors<T, ast::moore_8_neighbors>, ast::constant<Z>>> {
    static constexpr int value = 1;
};
template <class Dict, class T, auto Z>
struct signal_width<Dict, ast::greater_than<ast::count_neighbors<T, ast::von_neumann_4_neighbors>, ast::constant<Z>>> {
    static constexpr int value = 1;
};

template <class Dict, class L>
struct signal_layout;
template <class Dict, class... Ss>
struct signal_layout<Dict, tlist<Ss...>> {
    static constexpr int total = (0 + ... + signal_width<Dict, Ss>::value);
    template <class S>
    static constexpr int offset() {
        int off = 0, found = -1;
        ((found = (std::is_same_v<S, Ss> && found < 0) ? off : found, off += signal_width<Dict, Ss>::value), ...);
        return found;
    }
};

// Truth-table pattern of variable j (0..4) in a 32-bit word; variable 5 is
// constant within one half of a 64-entry table.
CB_HD constexpr word var_pattern(int j, int half) {
    constexpr word pat[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
    return j < 5 ? pat[j] : (half ? ~word(0) : word(0));
}

// Counts of a fixed state enter a synthesised network unfinished: the network
// receives the carry-save halves of the count, and the last additions become
// part of the network's own LOP3s.
//   Moore: low = a.s3 + b.s3 + m.s2 and high = a.c3 + b.c3 + m.c2 (each 0..3,
//     two planes: xor3 and maj3), count = low + 2 high -- four LOP3s where
//     the binary count (lower<count_neighbors<...>> above) takes eight;
//   von Neumann: low = u + d + m.s2 (xor3, maj3) and m.c2, count = low +
//     2 m.c2 -- two LOP3s where the binary count takes four.
// The symbolic context adds the halves back into the binary count on
// truth-table patterns, so the rule sees the same count.
template <class S>
struct packed_count : std::false_type {};
template <auto V>
struct packed_count<ast::count_neighbors<ast::state_constant<V>, ast::moore_8_neighbors>> : std::true_type {
    CB_HD static constexpr planes<4> binary(const word* x) {  // x: low0, low1, high0, high1
        const word c1 = x[1] & x[2];
        return planes<4>{{x[0], word(x[1] ^ x[2]), word(x[3] ^ c1), word(x[3] & c1)}};
    }
};
template <auto V>
struct packed_count<ast::count_neighbors<ast::state_constant<V>, ast::von_neumann_4_neighbors>> : std::true_type {
    CB_HD static constexpr planes<3> binary(const word* x) {  // x: low0, low1, m.c2
        return planes<3>{{x[0], word(x[1] ^ x[2]), word(x[1] & x[2])}};
    }
};

template <class Dict, class Targets, class S>
struct packed_signal;
template <class Dict, class Targets, auto V>
struct packed_signal<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::moore_8_neighbors>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class C>
    CB_HD static planes<4> eval(const C& c) {
        const count_cache& a = c.up.cc[slot];
        const count_cache& b = c.dn.cc[slot];
        const count_cache& m = c.mid.cc[slot];
        return planes<4>{{xor3(a.s3, b.s3, m.s2), maj3(a.s3, b.s3, m.s2), xor3(a.c3, b.c3, m.c2),
                          maj3(a.c3, b.c3, m.c2)}};
    }
};
template <class Dict, class Targets, auto V>
struct packed_signal<Dict, Targets, ast::count_neighbors<ast::state_constant<V>, ast::von_neumann_4_neighbors>> {
    static constexpr int slot = iindex<Targets, Dict::state_to_index(V)>::value;
    template <class C>
    CB_HD static planes<3> eval(const C& c) {
        const word u = c.up.cc[slot].P[1], d = c.dn.cc[slot].P[1];
        const count_cache& m = c.mid.cc[slot];
        return planes<3>{{xor3(u, d, m.s2), maj3(u, d, m.s2), m.c2}};
    }
};

// Symbolic evaluation context: signal S yields planes of variable patterns.
template <class Dict, class Signals, int TP, int HALF>
struct sym_ctx {
    static constexpr int tp = TP;
    static constexpr bool symbolic = true;
    template <class S>
    constexpr auto sig() const {
        constexpr int off = signal_layout<Dict, Signals>::template offset<S>();
        constexpr int w = signal_width<Dict, S>::value;
        if constexpr (packed_count<S>::value) {
            word x[w] = {};
            for (int i = 0; i < w; ++i) x[i] = var_pattern(off + i, HALF);
            return packed_count<S>::binary(x);
        } else if constexpr (w == 1 && !std::is_same_v<S, ast::neighbor_at<0, 0>> &&
                             !std::is_same_v<S, ast::margolus_180_neighbor>) {
            return var_pattern(off, HALF);  // a condition
        } else {
            planes<w> r{};
            for (int i = 0; i < w; ++i) r.p[i] = var_pattern(off + i, HALF);
            return r;
        }
    }
};

using tt_t = unsigned long long;

struct lop_node {
    int a, b, c;  // value indices: 0..n-1 inputs, n.. nodes, CONST0 / CONST1
    int imm;      // LOP3 immediate: f(0xF0, 0xCC, 0xAA)
};

constexpr int SYNTH_MAX_NODES = 64;
constexpr int CONST0 = -1, CONST1 = -2;

struct lop_net {
    int n = 0;       // input variables
    int nn = 0;      // nodes
    int nout = 0;    // outputs
    bool ok = true;  // false: node budget exceeded
    lop_node nodes[SYNTH_MAX_NODES] = {};
    tt_t node_tt[SYNTH_MAX_NODES] = {};
    int out[MAX_OUT_PLANES] = {};
};

constexpr tt_t tt_mask(int n) { return n >= 6 ? ~tt_t(0) : ((tt_t(1) << (1 << n)) - 1); }
// bit m of variable j's table = bit j of m, for up to six variables
constexpr tt_t tt_var(int j, int n) {
    constexpr tt_t pat[6] = {0xAAAAAAAAAAAAAAAAull, 0xCCCCCCCCCCCCCCCCull, 0xF0F0F0F0F0F0F0F0ull,
                             0xFF00FF00FF00FF00ull, 0xFFFF0000FFFF0000ull, 0xFFFFFFFF00000000ull};
    return pat[j] & tt_mask(n);
}
constexpr tt_t tt_cof(tt_t t, int v, int val, int n) {
    const tt_t pv = tt_var(v, n);
    const int sh = 1 << v;
    if (val) {
        const tt_t hi = t & pv;
        return (hi | (hi >> sh)) & tt_mask(n);
    }
    const tt_t lo = t & ~pv & tt_mask(n);
    return (lo | (lo << sh)) & tt_mask(n);
}
constexpr int tt_support(tt_t t, int n) {
    int s = 0;
    for (int v = 0; v < n; ++v)
        if (tt_cof(t, v, 0, n) != tt_cof(t, v, 1, n)) s |= 1 << v;
    return s;
}
constexpr int popc(int x) {
    int c = 0;
    for (; x; x &= x - 1) ++c;
    return c;
}

// Estimated node count of a function (Shannon with leaves of <= 3 variables).
constexpr int tt_cost(tt_t t, int n, int depth = 0) {
    const tt_t m = tt_mask(n);
    t &= m;
    if (t == 0 || t == m) return 0;
    const int s = tt_support(t, n);
    if (popc(s) == 1) {
        for (int v = 0; v < n; ++v)
            if (s == (1 << v) && t == tt_var(v, n)) return 0;
        return 1;
    }
    if (popc(s) <= 3) return 1;
    if (depth > 4) return 99;
    int best = 999;
    for (int v = 0; v < n; ++v)
        if ((s >> v) & 1) {
            const int c = 1 + tt_cost(tt_cof(t, v, 0, n), n, depth + 1) + tt_cost(tt_cof(t, v, 1, n), n, depth + 1);
            if (c < best) best = c;
        }
    return best;
}

// Truth table of a value index (input, node or constant).
constexpr tt_t value_tt(const lop_net& net, int idx) {
    if (idx == CONST0) return 0;
    if (idx == CONST1) return tt_mask(net.n);
    if (idx < net.n) return tt_var(idx, net.n);
    return net.node_tt[idx - net.n];
}

// 8-bit LOP3 operand pattern of a value used at operand slot `slot` (0xF0,
// 0xCC, 0xAA), or of a constant.
constexpr int operand_pattern(int idx, int slot) {
    if (idx == CONST0) return 0x00;
    if (idx == CONST1) return 0xFF;
    return slot == 0 ? 0xF0 : (slot == 1 ? 0xCC : 0xAA);
}

constexpr int add_node(lop_net& net, int a, int b, int c, int imm, tt_t t) {
    for (int i = 0; i < net.nn; ++i)
        if (net.node_tt[i] == t) return net.n + i;
    if (net.nn >= SYNTH_MAX_NODES) {
        net.ok = false;
        return CONST0;
    }
    // constant operands are folded into the immediate; give them a real register
    net.nodes[net.nn] = lop_node{a < 0 ? 0 : a, b < 0 ? 0 : b, c < 0 ? 0 : c, imm & 0xFF};
    net.node_tt[net.nn] = t;
    return net.n + net.nn++;
}

constexpr int emit(lop_net& net, tt_t t) {
    const int n = net.n;
    const tt_t m = tt_mask(n);
    t &= m;
    if (t == 0) return CONST0;
    if (t == m) return CONST1;
    for (int v = 0; v < n; ++v)
        if (t == tt_var(v, n)) return v;
    for (int i = 0; i < net.nn; ++i)
        if (net.node_tt[i] == t) return n + i;
    const int s = tt_support(t, n);
    if (popc(s) <= 3) {
        int vars[3] = {0, 0, 0}, k = 0;
        for (int v = 0; v < n && k < 3; ++v)
            if ((s >> v) & 1) vars[k++] = v;
        int imm = 0;
        for (int bit = 0; bit < 8; ++bit) {
            const int xa = (bit >> 2) & 1, xb = (bit >> 1) & 1, xc = bit & 1;
            int mt = 0;
            if (k > 0 && xa) mt |= 1 << vars[0];
            if (k > 1 && xb) mt |= 1 << vars[1];
            if (k > 2 && xc) mt |= 1 << vars[2];
            if ((t >> mt) & 1) imm |= 1 << bit;
        }
        return add_node(net, vars[0], vars[1], vars[2], imm, t);
    }
    // Shannon split on the variable with the cheapest cofactors
    int best_v = -1, best_c = 1 << 20;
    for (int v = 0; v < n; ++v)
        if ((s >> v) & 1) {
            const int c = tt_cost(tt_cof(t, v, 0, n), n) + tt_cost(tt_cof(t, v, 1, n), n);
            if (c < best_c) best_c = c, best_v = v;
        }
    const int i0 = emit(net, tt_cof(t, best_v, 0, n));
    const int i1 = emit(net, tt_cof(t, best_v, 1, n));
    // v ? i1 : i0
    const int pv = 0xF0, p1 = operand_pattern(i1, 1), p0 = operand_pattern(i0, 2);
    const int imm = (pv & p1) | (~pv & p0);
    return add_node(net, best_v, i1, i0, imm, t);
}

// The synthesised network of rule E at step parity TP (ok == false when the
// rule has more than 6 signal bits or the node budget overflows).
template <class Dict, class Targets, class E, int TP>
struct synth {
    using signals = typename signals_of<E, TP>::type;
    using layout = signal_layout<Dict, signals>;
    static constexpr int n = layout::total;
    static constexpr int NB = Dict::needed_bits;

    template <int HALF>
    static constexpr auto table_half() {
        return as_planes(ev<Dict, Targets, E>(sym_ctx<Dict, signals, TP, HALF>{}));
    }

    static constexpr lop_net build() {
        lop_net net;
        if (n > 6 || n < 1) {
            net.ok = false;
            return net;
        }
        net.n = n;
        net.nout = NB;
        constexpr auto lo = table_half<0>();
        constexpr auto hi = table_half<1>();
        constexpr int B = decltype(lo)::width;
        tt_t tts[MAX_OUT_PLANES] = {};
        for (int p = 0; p < NB; ++p) {
            if (p >= B) {
                tts[p] = 0;
                continue;
            }
            const tt_t l = lo.p[p < B ? p : 0], h = hi.p[p < B ? p : 0];
            tts[p] = n <= 5 ? (tt_t(l) & tt_mask(n)) : (tt_t(l) | (tt_t(h) << 32));
        }
        for (int p = 0; p < NB; ++p) net.out[p] = emit(net, tts[p]);
        return net;
    }
    static constexpr lop_net net = build();
    static constexpr bool ok = net.ok;
};

template <int IMM>
CB_HD word lop3(word a, word b, word c) {
#if defined(__CUDA_ARCH__)
    word d;
    asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(IMM));
    return d;
#else
    word r = 0;
    for (int k = 0; k < 8; ++k)
        if ((IMM >> k) & 1) r |= (((k >> 2) & 1) ? a : ~a) & (((k >> 1) & 1) ? b : ~b) & ((k & 1) ? c : ~c);
    return r;
#endif
}

template <const lop_net& NET, int I>
CB_HD void run_node(word* v) {
    constexpr lop_node nd = NET.nodes[I];
    v[NET.n + I] = lop3<nd.imm>(v[nd.a], v[nd.b], v[nd.c]);
}

template <const lop_net& NET, std::size_t... I>
CB_HD void run_net(word* v, std::index_sequence<I...>) {
    (run_node<NET, (int)I>(v), ...);
}

// ------------------------------------------------------------------ a rule
// rule_net<Dict, Rule>: the lowered rule.  eval() returns the NB planes of
// the next state of 32 cells; narrower results are zero-extended, wider ones
// truncated to the stored planes (the extra planes of a valid state are zero).
template <class Dict, class Rule>
struct rule_net {
    static constexpr int NB = Dict::needed_bits;
    using targets = targets_of<Dict, Rule>;
    using feat = row_feat<NB, targets>;
    using preds_t = pred_set<targets>;
    static constexpr bool need_shift = uses_shift<Rule>::value;
    static constexpr bool need_sums = uses_sums<Rule>::value;
    static constexpr bool need_any = uses_any<Rule>::value;

    CB_HD static preds_t preds(const word* C) { return preds_of_impl<NB>(C, targets{}); }

    // features of one word given its neighbours' predicates
    CB_HD static feat make(const word* C, const word* L, const word* R, const preds_t& pc, const preds_t& pl,
                           const preds_t& pr) {
        return make_row_feat<NB, targets, need_shift, need_sums, need_any>(C, L, R, pc, pl, pr);
    }

    // features of one word from its own and its two neighbour words
    CB_HD static feat make_feat(const word* C, const word* L, const word* R) {
        return make(C, L, R, preds(C), preds(L), preds(R));
    }

    template <int TP>
    CB_HD static void eval(const feat& up, const feat& mid, const feat& dn, int ypar, word* out) {
        const ctx<feat, TP> c{up, mid, dn, ypar};
        using S = synth<Dict, targets, Rule, TP>;
        if constexpr (S::ok) {
            // signals through the generic lowering, then the LOP3 network
            word v[S::net.n + S::net.nn + 1];
            fill_signals<TP>(c, v, typename S::signals{});
            run_net<S::net>(v, std::make_index_sequence<S::net.nn>{});
            store_outputs<S::net>(v, out, std::make_index_sequence<NB>{});
        } else {
            const auto r = as_planes(ev<Dict, targets, Rule>(c));
            constexpr int B = decltype(r)::width;
#pragma unroll
            for (int p = 0; p < NB; ++p) out[p] = p < B ? r.p[p < B ? p : 0] : word(0);
        }
    }

    // network size (0 when the rule is evaluated by the generic lowering)
    template <int TP>
    static constexpr int synthesized_nodes() {
        using S = synth<Dict, targets, Rule, TP>;
        return S::ok ? S::net.nn : -1;
    }

  private:
    template <const lop_net& NET, std::size_t... P>
    CB_HD static void store_outputs(const word* v, word* out, std::index_sequence<P...>) {
        (
            [&] {
                constexpr int idx = NET.out[P];
                if constexpr (idx == CONST0)
                    out[P] = 0;
                else if constexpr (idx == CONST1)
                    out[P] = ~word(0);
                else
                    out[P] = v[idx];
            }(),
            ...);
    }

    template <class S, class C>
    CB_HD static auto signal_value(const C& c) {
        if constexpr (packed_count<S>::value)
            return packed_signal<Dict, targets, S>::eval(c);  // the network finishes the count
        else
            return as_planes(ev<Dict, targets, S>(c));
    }

    template <int TP, class C, class... Ss>
    CB_HD static void fill_signals(const C& c, word* v, tlist<Ss...>) {
        using L = signal_layout<Dict, tlist<Ss...>>;
        (
            [&] {
                const auto s = signal_value<Ss>(c);
                constexpr int off = L::template offset<Ss>();
#pragma unroll
                for (int i = 0; i < decltype(s)::width; ++i) v[off + i] = s.p[i];
            }(),
            ...);
    }
};

}  // namespace cellato::b200

#endif  // CELLATO_B200_LOWER_CUH
