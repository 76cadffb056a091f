// Minimal std-based stand-in for the handful of Boost metaprogramming names
// that the MTL4/ITL sparse-solve headers use (boost::mpl::bool_/int_/if_/...,
// boost::is_same and friends, enable_if, shared_ptr, tuple).  Boost itself is
// not installed on this machine; none of these names carries arithmetic, so a
// restatement in terms of <type_traits>, <memory> and <tuple> lets the
// unmodified reference headers compile for use as a CPU test oracle.
//
// TEST INFRASTRUCTURE ONLY: nothing in the shipped library includes this file.
// Written from the C++ standard library's vocabulary; every forwarding header
// oracle/_ref/compat/boost/<name>.hpp (generated by oracle/Makefile) includes
// just this file.
#ifndef MTLGPU_ORACLE_BOOST_COMPAT_HPP
#define MTLGPU_ORACLE_BOOST_COMPAT_HPP

#include <cstddef>
#include <memory>
#include <tuple>
#include <type_traits>
#include <unordered_set>
#include <algorithm>
#include <complex>
#include <climits>
#include <cassert>
#include <unordered_map>

#define BOOST_STATIC_ASSERT(...) static_assert((__VA_ARGS__), #__VA_ARGS__)
#define BOOST_STATIC_ASSERT_MSG(c, m) static_assert((c), m)
#define BOOST_MPL_ASSERT(p) static_assert(p::value, #p)
#define BOOST_ASSERT(e) assert(e)

namespace boost {

namespace mpl {
struct void_ { typedef void_ type; };
struct na {};

template <bool B> struct bool_ : std::integral_constant<bool, B> {
  typedef bool_ type;
  typedef bool value_type;
};
typedef bool_<true> true_;
typedef bool_<false> false_;

template <int N> struct int_ : std::integral_constant<int, N> {
  typedef int_ type;
  typedef int value_type;
  typedef int_<N + 1> next;
  typedef int_<N - 1> prior;
};
template <long N> struct long_ : std::integral_constant<long, N> {
  typedef long_ type;
};
template <std::size_t N> struct size_t : std::integral_constant<std::size_t, N> {
  typedef size_t type;
};
template <typename T, T N> struct integral_c : std::integral_constant<T, N> {
  typedef integral_c type;
};

template <bool C, typename T, typename F> struct if_c { typedef T type; };
template <typename T, typename F> struct if_c<false, T, F> { typedef F type; };
template <typename C, typename T, typename F> struct if_ : if_c<bool(C::value), T, F> {};

template <typename C, typename F1, typename F2>
struct eval_if : if_<C, F1, F2>::type {};
template <bool C, typename F1, typename F2>
struct eval_if_c : if_c<C, F1, F2>::type {};

// and_/or_ short-circuit like Boost's: later arguments are not instantiated
// once the result is known (std::conjunction/std::disjunction do the same).
template <typename... T> struct and_ : bool_<std::conjunction<T...>::value> {};
template <typename... T> struct or_ : bool_<std::disjunction<T...>::value> {};
template <typename T> struct not_ : bool_<!T::value> {};

template <typename A, typename B> struct less : bool_<(A::value < B::value)> {};
template <typename A, typename B> struct less_equal : bool_<(A::value <= B::value)> {};
template <typename A, typename B> struct greater : bool_<(A::value > B::value)> {};
template <typename A, typename B> struct greater_equal : bool_<(A::value >= B::value)> {};
template <typename A, typename B> struct equal_to : bool_<(A::value == B::value)> {};
template <typename A, typename B> struct max : if_c<(A::value < B::value), B, A>::type {};
template <typename A, typename B> struct min : if_c<(B::value < A::value), B, A>::type {};
template <typename A, typename B> struct plus : integral_c<decltype(A::value + B::value), A::value + B::value> {};
template <typename A, typename B> struct minus : integral_c<decltype(A::value - B::value), A::value - B::value> {};

// --- pair / map: a compile-time association list -------------------------
template <typename K, typename V> struct pair {
  typedef pair type;
  typedef K first;
  typedef V second;
};
template <typename... P> struct map { typedef map type; };

namespace compat_detail {
template <typename Map, typename Key> struct map_at;
template <typename Key> struct map_at<map<>, Key> { typedef void_ type; };
template <typename K, typename V, typename... Rest, typename Key>
struct map_at<map<pair<K, V>, Rest...>, Key> : map_at<map<Rest...>, Key> {};
template <typename K, typename V, typename... Rest>
struct map_at<map<pair<K, V>, Rest...>, K> { typedef V type; };

template <typename Map, typename Key> struct map_erase;
template <typename Key> struct map_erase<map<>, Key> { typedef map<> type; };
template <typename Head, typename... Rest, typename Key>
struct map_erase<map<Head, Rest...>, Key> {
  typedef typename map_erase<map<Rest...>, Key>::type tail;
  template <typename T> struct prepend;
  template <typename... P> struct prepend<map<P...>> { typedef map<Head, P...> type; };
  typedef typename std::conditional<std::is_same<typename Head::first, Key>::value, tail,
                                    typename prepend<tail>::type>::type type;
};

template <typename Seq, std::size_t N> struct seq_at;
}  // namespace compat_detail

template <typename Seq, typename Key> struct at;
template <typename... P, typename Key>
struct at<map<P...>, Key> { typedef typename compat_detail::map_at<map<P...>, Key>::type type; };

template <typename Map, typename Key> struct erase_key {
  typedef typename compat_detail::map_erase<Map, Key>::type type;
};

template <typename Map, typename PosOrPair, typename Pair = na> struct insert;
template <typename... P, typename Pos, typename K, typename V>
struct insert<map<P...>, Pos, pair<K, V>> {
  typedef map<pair<K, V>, P...> type;
};
template <typename... P, typename K, typename V>
struct insert<map<P...>, pair<K, V>, na> {
  typedef map<pair<K, V>, P...> type;
};

// vector-like sequence, indexed by at_c
template <typename... T> struct vector { typedef vector type; };
template <typename Seq, int N> struct at_c;
template <typename H, typename... T> struct at_c<vector<H, T...>, 0> { typedef H type; };
template <typename H, typename... T, int N>
struct at_c<vector<H, T...>, N> : at_c<vector<T...>, N - 1> {};
}  // namespace mpl

// --- type traits ----------------------------------------------------------
// Boost's traits convert to mpl::bool_, which MTL relies on for overload
// dispatch (e.g. functions taking boost::mpl::true_ / boost::mpl::false_).
template <typename T, T V> struct integral_constant : std::integral_constant<T, V> {
  typedef integral_constant type;
};
template <bool V> struct integral_constant<bool, V> : mpl::bool_<V> {
  typedef integral_constant type;
};
typedef integral_constant<bool, true> true_type;
typedef integral_constant<bool, false> false_type;

#define MTLGPU_COMPAT_BOOL_TRAIT1(name) \
  template <typename T> struct name : integral_constant<bool, std::name<T>::value> {};
#define MTLGPU_COMPAT_BOOL_TRAIT2(name) \
  template <typename T, typename U> struct name : integral_constant<bool, std::name<T, U>::value> {};
MTLGPU_COMPAT_BOOL_TRAIT2(is_same)
MTLGPU_COMPAT_BOOL_TRAIT2(is_base_of)
MTLGPU_COMPAT_BOOL_TRAIT2(is_convertible)
MTLGPU_COMPAT_BOOL_TRAIT1(is_integral)
MTLGPU_COMPAT_BOOL_TRAIT1(is_unsigned)
MTLGPU_COMPAT_BOOL_TRAIT1(is_signed)
MTLGPU_COMPAT_BOOL_TRAIT1(is_const)
MTLGPU_COMPAT_BOOL_TRAIT1(is_volatile)
MTLGPU_COMPAT_BOOL_TRAIT1(is_floating_point)
MTLGPU_COMPAT_BOOL_TRAIT1(is_arithmetic)
MTLGPU_COMPAT_BOOL_TRAIT1(is_scalar)
MTLGPU_COMPAT_BOOL_TRAIT1(is_empty)
MTLGPU_COMPAT_BOOL_TRAIT1(is_pointer)
MTLGPU_COMPAT_BOOL_TRAIT1(is_reference)
MTLGPU_COMPAT_BOOL_TRAIT1(is_fundamental)
MTLGPU_COMPAT_BOOL_TRAIT1(is_class)
#undef MTLGPU_COMPAT_BOOL_TRAIT1
#undef MTLGPU_COMPAT_BOOL_TRAIT2

template <typename T> struct is_complex : false_type {};
template <typename T> struct is_complex<std::complex<T>> : true_type {};
template <typename T> struct is_complex<const T> : is_complex<T> {};

template <typename T> struct remove_const { typedef typename std::remove_const<T>::type type; };
template <typename T> struct remove_reference { typedef typename std::remove_reference<T>::type type; };
template <typename T> struct remove_cv { typedef typename std::remove_cv<T>::type type; };
template <typename T> struct remove_pointer { typedef typename std::remove_pointer<T>::type type; };
template <typename T> struct add_const { typedef typename std::add_const<T>::type type; };
template <typename T> struct add_reference { typedef typename std::add_lvalue_reference<T>::type type; };
template <typename T> struct add_pointer { typedef typename std::add_pointer<T>::type type; };
template <typename T> struct make_signed { typedef typename std::make_signed<T>::type type; };
template <typename T> struct make_unsigned { typedef typename std::make_unsigned<T>::type type; };

// --- enable_if family -----------------------------------------------------
template <bool B, typename T = void> struct enable_if_c { typedef T type; };
template <typename T> struct enable_if_c<false, T> {};
template <typename C, typename T = void> struct enable_if : enable_if_c<bool(C::value), T> {};
template <bool B, typename T = void> struct disable_if_c { typedef T type; };
template <typename T> struct disable_if_c<true, T> {};
template <typename C, typename T = void> struct disable_if : disable_if_c<bool(C::value), T> {};
template <bool B, typename F> struct lazy_enable_if_c { typedef typename F::type type; };
template <typename F> struct lazy_enable_if_c<false, F> {};
template <typename C, typename F> struct lazy_enable_if : lazy_enable_if_c<bool(C::value), F> {};
template <bool B, typename F> struct lazy_disable_if_c { typedef typename F::type type; };
template <typename F> struct lazy_disable_if_c<true, F> {};
template <typename C, typename F> struct lazy_disable_if : lazy_disable_if_c<bool(C::value), F> {};

// --- smart pointer / tuple ------------------------------------------------
using std::shared_ptr;
using std::make_shared;
using std::tuple;
using std::tie;
using std::make_tuple;
using std::get;
template <typename T, typename H = std::hash<T>, typename E = std::equal_to<T>>
using unordered_set = std::unordered_set<T, H, E>;

template <typename K, typename V, typename H = std::hash<K>, typename E = std::equal_to<K>>
using unordered_map = std::unordered_map<K, V, H, E>;

template <typename Target, typename Source> inline Target numeric_cast(Source s) {
  return static_cast<Target>(s);
}

namespace tuples {
using std::tuple;
using std::get;
}  // namespace tuples
}  // namespace boost

#endif  // MTLGPU_ORACLE_BOOST_COMPAT_HPP
