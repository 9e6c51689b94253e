// Project-written stand-in for the small part of Boost.Multiprecision that the
// reference's CPU sources use (cpp_int, int128_t, msb, divide_qr).  It exists
// only so that the reference's exact CPU lane can be compiled here as a test
// oracle; Boost itself is not installed.  Semantics follow Boost's documented
// behaviour for signed-magnitude cpp_int: truncating division, remainder with
// the sign of the dividend, arbitrary precision.
//
// Storage: sign + magnitude in 64-bit limbs with four limbs inline, so values
// up to 256 bits never touch the heap.
#pragma once

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <limits>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

namespace boost {
namespace multiprecision {

namespace shim_detail {
using limb = std::uint64_t;
using dlimb = unsigned __int128;
}  // namespace shim_detail

class cpp_int {
  using limb = shim_detail::limb;
  using dlimb = shim_detail::dlimb;
  static constexpr unsigned inline_cap = 4;

 public:
  cpp_int() noexcept : size_(0), cap_(inline_cap), neg_(false), heap_(nullptr) {}
  ~cpp_int() { delete[] heap_; }

  cpp_int(const cpp_int& o) : cpp_int() { assign_mag(o.data(), o.size_); neg_ = o.neg_; }
  cpp_int(cpp_int&& o) noexcept : cpp_int() { steal(o); }
  cpp_int& operator=(const cpp_int& o) {
    if (this != &o) { assign_mag(o.data(), o.size_); neg_ = o.neg_; }
    return *this;
  }
  cpp_int& operator=(cpp_int&& o) noexcept {
    if (this != &o) { delete[] heap_; heap_ = nullptr; cap_ = inline_cap; size_ = 0; steal(o); }
    return *this;
  }

  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
  cpp_int(T v) : cpp_int() { set_integral(v); }
  cpp_int(__int128 v) : cpp_int() { set_i128(v); }
  cpp_int(unsigned __int128 v) : cpp_int() { set_u128(v, false); }
  explicit cpp_int(double v) : cpp_int() { set_double(v); }
  explicit cpp_int(const char* text) : cpp_int() { set_string(text); }
  explicit cpp_int(const std::string& text) : cpp_int() { set_string(text.c_str()); }

  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>
  cpp_int& operator=(T v) { set_integral(v); return *this; }

  // ---- observers -------------------------------------------------------
  int sign() const noexcept { return size_ == 0 ? 0 : (neg_ ? -1 : 1); }
  bool is_zero() const noexcept { return size_ == 0; }
  explicit operator bool() const noexcept { return size_ != 0; }

  std::string str(std::streamsize = 0, std::ios_base::fmtflags = std::ios_base::fmtflags(0)) const {
    if (size_ == 0) return "0";
    cpp_int t = *this;
    t.neg_ = false;
    std::string digits;
    const limb chunk = 10000000000000000000ULL;  // 10^19
    while (t.size_ != 0) {
      limb rem = t.div_small_inplace(chunk);
      for (int i = 0; i < 19; ++i) {
        digits.push_back(char('0' + rem % 10));
        rem /= 10;
        if (t.size_ == 0 && rem == 0) break;
      }
    }
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    if (neg_) digits.push_back('-');
    std::reverse(digits.begin(), digits.end());
    return digits;
  }

  template <typename T>
  T convert_to() const {
    if constexpr (std::is_floating_point<T>::value) {
      long double r = 0;
      for (unsigned i = size_; i-- > 0;) r = r * 18446744073709551616.0L + (long double)data()[i];
      return static_cast<T>(neg_ ? -r : r);
    } else {
      static_assert(std::is_integral<T>::value, "convert_to supports integral and floating types");
      using U = typename std::make_unsigned<T>::type;
      unsigned __int128 m = 0;
      if (size_ > 0) m = data()[0];
      if (size_ > 1) m |= (unsigned __int128)data()[1] << 64;
      bool big = size_ > 2;
      if constexpr (std::is_signed<T>::value) {
        const unsigned __int128 lim = (unsigned __int128)(U)std::numeric_limits<T>::max();
        if (!neg_) return (big || m > lim) ? std::numeric_limits<T>::max() : (T)m;
        if (big || m > lim + 1) return std::numeric_limits<T>::min();
        return (T)(-(__int128)m);
      } else {
        if (neg_) return 0;
        const unsigned __int128 lim = (U)std::numeric_limits<U>::max();
        return (big || m > lim) ? std::numeric_limits<T>::max() : (T)m;
      }
    }
  }
  template <typename T, typename std::enable_if<std::is_arithmetic<T>::value, int>::type = 0>
  explicit operator T() const { return convert_to<T>(); }

  // ---- arithmetic -------------------------------------------------------
  friend cpp_int operator-(const cpp_int& a) { cpp_int r = a; if (r.size_) r.neg_ = !r.neg_; return r; }
  friend cpp_int operator-(cpp_int&& a) { if (a.size_) a.neg_ = !a.neg_; return std::move(a); }
  friend const cpp_int& operator+(const cpp_int& a) { return a; }

  cpp_int& operator+=(const cpp_int& b) { add_signed(b, false); return *this; }
  cpp_int& operator-=(const cpp_int& b) { add_signed(b, true); return *this; }
  cpp_int& operator*=(const cpp_int& b) { *this = mul(*this, b); return *this; }
  cpp_int& operator/=(const cpp_int& b) { cpp_int q, r; divmod(*this, b, q, r); *this = std::move(q); return *this; }
  cpp_int& operator%=(const cpp_int& b) { cpp_int q, r; divmod(*this, b, q, r); *this = std::move(r); return *this; }
  cpp_int& operator<<=(unsigned long long s) { shl(s); return *this; }
  cpp_int& operator>>=(unsigned long long s) { shr(s); return *this; }
  cpp_int& operator&=(const cpp_int& b) { bitop(b, 0); return *this; }
  cpp_int& operator|=(const cpp_int& b) { bitop(b, 1); return *this; }
  cpp_int& operator^=(const cpp_int& b) { bitop(b, 2); return *this; }
  cpp_int& operator++() { return *this += cpp_int(1); }
  cpp_int& operator--() { return *this -= cpp_int(1); }
  cpp_int operator++(int) { cpp_int t = *this; ++*this; return t; }
  cpp_int operator--(int) { cpp_int t = *this; --*this; return t; }

  friend cpp_int operator+(cpp_int a, const cpp_int& b) { a += b; return a; }
  friend cpp_int operator-(cpp_int a, const cpp_int& b) { a -= b; return a; }
  friend cpp_int operator*(const cpp_int& a, const cpp_int& b) { return mul(a, b); }
  friend cpp_int operator/(const cpp_int& a, const cpp_int& b) { cpp_int q, r; divmod(a, b, q, r); return q; }
  friend cpp_int operator%(const cpp_int& a, const cpp_int& b) { cpp_int q, r; divmod(a, b, q, r); return r; }
  friend cpp_int operator&(cpp_int a, const cpp_int& b) { a &= b; return a; }
  friend cpp_int operator|(cpp_int a, const cpp_int& b) { a |= b; return a; }
  friend cpp_int operator^(cpp_int a, const cpp_int& b) { a ^= b; return a; }
  template <typename S, typename std::enable_if<std::is_integral<S>::value, int>::type = 0>
  friend cpp_int operator<<(cpp_int a, S s) { a.shl((unsigned long long)s); return a; }
  template <typename S, typename std::enable_if<std::is_integral<S>::value, int>::type = 0>
  friend cpp_int operator>>(cpp_int a, S s) { a.shr((unsigned long long)s); return a; }

  // mixed integral operands
#define SHIM_MIXED(op)                                                                            \
  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>       \
  friend cpp_int operator op(const cpp_int& a, T b) { return a op cpp_int(b); }                   \
  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>       \
  friend cpp_int operator op(T a, const cpp_int& b) { return cpp_int(a) op b; }
  SHIM_MIXED(+) SHIM_MIXED(-) SHIM_MIXED(*) SHIM_MIXED(/) SHIM_MIXED(%) SHIM_MIXED(&) SHIM_MIXED(|) SHIM_MIXED(^)
#undef SHIM_MIXED
#define SHIM_MIXED_ASSIGN(op)                                                                     \
  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>       \
  cpp_int& operator op(T b) { return *this op cpp_int(b); }
  SHIM_MIXED_ASSIGN(+=) SHIM_MIXED_ASSIGN(-=) SHIM_MIXED_ASSIGN(*=) SHIM_MIXED_ASSIGN(/=) SHIM_MIXED_ASSIGN(%=)
#undef SHIM_MIXED_ASSIGN

  // ---- comparison -------------------------------------------------------
  static int compare(const cpp_int& a, const cpp_int& b) noexcept {
    if (a.neg_ != b.neg_ && (a.size_ | b.size_)) return a.neg_ ? -1 : 1;
    int c = cmp_mag(a.data(), a.size_, b.data(), b.size_);
    return a.neg_ ? -c : c;
  }
#define SHIM_CMP(op)                                                                              \
  friend bool operator op(const cpp_int& a, const cpp_int& b) noexcept { return compare(a, b) op 0; } \
  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>       \
  friend bool operator op(const cpp_int& a, T b) { return compare(a, cpp_int(b)) op 0; }          \
  template <typename T, typename std::enable_if<std::is_integral<T>::value, int>::type = 0>       \
  friend bool operator op(T a, const cpp_int& b) { return compare(cpp_int(a), b) op 0; }
  SHIM_CMP(==) SHIM_CMP(!=) SHIM_CMP(<) SHIM_CMP(<=) SHIM_CMP(>) SHIM_CMP(>=)
#undef SHIM_CMP

  friend std::ostream& operator<<(std::ostream& os, const cpp_int& v) { return os << v.str(); }

  // ---- helpers used by free functions -------------------------------------
  unsigned long long msb_index() const {
    if (size_ == 0) throw std::domain_error("msb of zero is undefined");
    limb top = data()[size_ - 1];
    return (unsigned long long)(size_ - 1) * 64 + (63 - (unsigned)__builtin_clzll(top));
  }
  unsigned long long lsb_index() const {
    if (size_ == 0) throw std::domain_error("lsb of zero is undefined");
    for (unsigned i = 0; i < size_; ++i)
      if (data()[i]) return (unsigned long long)i * 64 + (unsigned)__builtin_ctzll(data()[i]);
    return 0;
  }
  bool test_bit(unsigned long long i) const {
    unsigned li = (unsigned)(i / 64);
    return li < size_ && ((data()[li] >> (i % 64)) & 1U);
  }
  static void divmod(const cpp_int& a, const cpp_int& b, cpp_int& q, cpp_int& r) {
    if (b.size_ == 0) throw std::overflow_error("Integer Division by zero.");
    const bool qneg = a.neg_ != b.neg_;
    const bool rneg = a.neg_;
    divmod_mag(a, b, q, r);
    q.neg_ = q.size_ ? qneg : false;
    r.neg_ = r.size_ ? rneg : false;
  }

 private:
  limb inline_[inline_cap];
  unsigned size_;
  unsigned cap_;
  bool neg_;
  limb* heap_;

  limb* data() noexcept { return heap_ ? heap_ : inline_; }
  const limb* data() const noexcept { return heap_ ? heap_ : inline_; }

  void steal(cpp_int& o) noexcept {
    neg_ = o.neg_;
    size_ = o.size_;
    if (o.heap_) {
      heap_ = o.heap_; cap_ = o.cap_;
      o.heap_ = nullptr; o.cap_ = inline_cap;
    } else {
      std::memcpy(inline_, o.inline_, sizeof(limb) * o.size_);
    }
    o.size_ = 0; o.neg_ = false;
  }
  void reserve(unsigned n) {
    if (n <= cap_) return;
    unsigned nc = std::max(n, cap_ * 2);
    limb* nh = new limb[nc];
    std::memcpy(nh, data(), sizeof(limb) * size_);
    delete[] heap_;
    heap_ = nh; cap_ = nc;
  }
  void trim() noexcept {
    const limb* d = data();
    while (size_ && d[size_ - 1] == 0) --size_;
    if (!size_) neg_ = false;
  }
  void assign_mag(const limb* src, unsigned n) {
    if (src == data()) { size_ = n; return; }
    size_ = 0;
    reserve(n);
    std::memmove(data(), src, sizeof(limb) * n);
    size_ = n;
  }
  template <typename T>
  void set_integral(T v) {
    if constexpr (std::is_signed<T>::value) set_i128((__int128)v);
    else set_u128((unsigned __int128)v, false);
  }
  void set_i128(__int128 v) {
    bool n = v < 0;
    unsigned __int128 m = n ? (unsigned __int128)0 - (unsigned __int128)v : (unsigned __int128)v;
    set_u128(m, n);
  }
  void set_u128(unsigned __int128 m, bool n) {
    size_ = 0;
    limb* d = data();
    d[0] = (limb)m; d[1] = (limb)(m >> 64);
    size_ = 2;
    neg_ = n;
    trim();
  }
  // decimal text with an optional leading '-' (hexadecimal "0x" accepted too)
  void set_string(const char* t) {
    size_ = 0; neg_ = false;
    bool n = false;
    if (*t == '-') { n = true; ++t; } else if (*t == '+') { ++t; }
    if (!*t) throw std::runtime_error("empty integer text");
    unsigned base = 10;
    if (t[0] == '0' && (t[1] == 'x' || t[1] == 'X')) { base = 16; t += 2; }
    for (; *t; ++t) {
      unsigned d;
      if (*t >= '0' && *t <= '9') d = unsigned(*t - '0');
      else if (base == 16 && *t >= 'a' && *t <= 'f') d = unsigned(*t - 'a' + 10);
      else if (base == 16 && *t >= 'A' && *t <= 'F') d = unsigned(*t - 'A' + 10);
      else throw std::runtime_error("unexpected character in integer text");
      *this = mul(*this, cpp_int(base));
      *this += cpp_int(d);
    }
    neg_ = n && size_;
  }
  void set_double(double v) {
    if (!(v == v) || v == std::numeric_limits<double>::infinity() || v == -std::numeric_limits<double>::infinity())
      throw std::domain_error("cannot convert a non-finite double to cpp_int");
    bool n = v < 0; if (n) v = -v;
    int e = 0;
    double f = __builtin_frexp(v, &e);  // v = f * 2^e, f in [0.5,1)
    if (v < 1.0) { size_ = 0; neg_ = false; return; }
    unsigned long long mant = (unsigned long long)__builtin_ldexp(f, 53);
    set_u128(mant, false);
    if (e >= 53) shl((unsigned long long)(e - 53)); else shr((unsigned long long)(53 - e));
    neg_ = n && size_;
  }

  static int cmp_mag(const limb* a, unsigned na, const limb* b, unsigned nb) noexcept {
    if (na != nb) return na < nb ? -1 : 1;
    for (unsigned i = na; i-- > 0;)
      if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
  }
  // this = |this| + |b|  (sign handled by caller)
  void add_mag(const limb* b, unsigned nb) {
    unsigned n = std::max(size_, nb);
    reserve(n + 1);
    limb* d = data();
    for (unsigned i = size_; i < n + 1; ++i) d[i] = 0;
    limb carry = 0;
    for (unsigned i = 0; i < n; ++i) {
      dlimb s = (dlimb)d[i] + (i < nb ? b[i] : 0) + carry;
      d[i] = (limb)s; carry = (limb)(s >> 64);
    }
    d[n] = carry;
    size_ = n + 1;
    bool n0 = neg_; trim(); if (size_) neg_ = n0;
  }
  // this = |this| - |b| where |this| >= |b|
  void sub_mag(const limb* b, unsigned nb) {
    limb* d = data();
    limb borrow = 0;
    for (unsigned i = 0; i < size_; ++i) {
      limb bi = i < nb ? b[i] : 0;
      dlimb s = (dlimb)d[i] - bi - borrow;
      d[i] = (limb)s;
      borrow = (limb)((s >> 64) & 1U);
    }
    bool n0 = neg_; trim(); if (size_) neg_ = n0;
  }
  void add_signed(const cpp_int& bref, bool negate_b) {
    if (bref.size_ == 0) return;
    cpp_int tmp;
    const cpp_int* bp = &bref;
    if (bp == this) { tmp = bref; bp = &tmp; }
    const bool bneg = negate_b ? !bp->neg_ : bp->neg_;
    if (size_ == 0) { assign_mag(bp->data(), bp->size_); neg_ = bneg; return; }
    if (neg_ == bneg) { add_mag(bp->data(), bp->size_); return; }
    int c = cmp_mag(data(), size_, bp->data(), bp->size_);
    if (c == 0) { size_ = 0; neg_ = false; return; }
    if (c > 0) { sub_mag(bp->data(), bp->size_); return; }
    cpp_int r = *bp; r.neg_ = bneg;
    r.sub_mag(data(), size_);
    *this = std::move(r);
  }
  static cpp_int mul(const cpp_int& a, const cpp_int& b) {
    cpp_int r;
    if (a.size_ == 0 || b.size_ == 0) return r;
    unsigned n = a.size_ + b.size_;
    r.reserve(n);
    limb* d = r.data();
    for (unsigned i = 0; i < n; ++i) d[i] = 0;
    const limb* ad = a.data(); const limb* bd = b.data();
    for (unsigned i = 0; i < a.size_; ++i) {
      limb carry = 0;
      const limb ai = ad[i];
      for (unsigned j = 0; j < b.size_; ++j) {
        dlimb t = (dlimb)ai * bd[j] + d[i + j] + carry;
        d[i + j] = (limb)t; carry = (limb)(t >> 64);
      }
      d[i + b.size_] = carry;
    }
    r.size_ = n;
    r.neg_ = a.neg_ != b.neg_;
    r.trim();
    return r;
  }
  // divide magnitude in place by a small divisor, return the remainder
  limb div_small_inplace(limb v) {
    limb* d = data();
    dlimb rem = 0;
    for (unsigned i = size_; i-- > 0;) {
      dlimb cur = (rem << 64) | d[i];
      d[i] = (limb)(cur / v);
      rem = cur % v;
    }
    bool n0 = neg_; trim(); if (size_) neg_ = n0;
    return (limb)rem;
  }
  // Knuth, TAOCP vol. 2, 4.3.1 algorithm D on 64-bit limbs (magnitudes only).
  static void divmod_mag(const cpp_int& a, const cpp_int& b, cpp_int& q, cpp_int& r) {
    if (cmp_mag(a.data(), a.size_, b.data(), b.size_) < 0) {
      cpp_int ra = a; ra.neg_ = false;
      q = cpp_int(); r = std::move(ra);
      return;
    }
    if (a.size_ <= 2) {  // both magnitudes fit 128 bits
      const limb* ad = a.data(); const limb* bd = b.data();
      const dlimb x = (dlimb)ad[0] | (a.size_ > 1 ? (dlimb)ad[1] << 64 : 0);
      const dlimb y = (dlimb)bd[0] | (b.size_ > 1 ? (dlimb)bd[1] << 64 : 0);
      cpp_int qq, rr;
      qq.set_u128(x / y, false);
      rr.set_u128(x % y, false);
      q = std::move(qq); r = std::move(rr);
      return;
    }
    if (b.size_ == 1) {
      cpp_int qa = a; qa.neg_ = false;
      limb rem = qa.div_small_inplace(b.data()[0]);
      q = std::move(qa);
      r = cpp_int(rem);
      return;
    }
    const unsigned n = b.size_, m = a.size_ - b.size_;
    const unsigned s = (unsigned)__builtin_clzll(b.data()[n - 1]);
    // normalised copies (on the stack for operands up to 32 limbs)
    constexpr unsigned kStackLimbs = 32;
    limb vbuf[kStackLimbs], ubuf[kStackLimbs + 1];
    const bool heap = n > kStackLimbs || a.size_ + 1 > kStackLimbs + 1;
    limb* vn = heap ? new limb[n] : vbuf;
    limb* un = heap ? new limb[a.size_ + 1] : ubuf;
    const limb* vb = b.data(); const limb* ua = a.data();
    for (unsigned i = n - 1; i > 0; --i)
      vn[i] = s ? (vb[i] << s) | (vb[i - 1] >> (64 - s)) : vb[i];
    vn[0] = vb[0] << s;
    un[a.size_] = s ? ua[a.size_ - 1] >> (64 - s) : 0;
    for (unsigned i = a.size_ - 1; i > 0; --i)
      un[i] = s ? (ua[i] << s) | (ua[i - 1] >> (64 - s)) : ua[i];
    un[0] = ua[0] << s;
    cpp_int qq; qq.reserve(m + 1); qq.size_ = m + 1;
    limb* qd = qq.data();
    for (unsigned jj = m + 1; jj-- > 0;) {
      const unsigned j = jj;
      dlimb num = ((dlimb)un[j + n] << 64) | un[j + n - 1];
      dlimb qhat = num / vn[n - 1];
      dlimb rhat = num % vn[n - 1];
      while (qhat >> 64 || qhat * vn[n - 2] > ((rhat << 64) | un[j + n - 2])) {
        --qhat; rhat += vn[n - 1];
        if (rhat >> 64) break;
      }
      // multiply and subtract
      limb borrow = 0, carry = 0;
      for (unsigned i = 0; i < n; ++i) {
        dlimb p = qhat * vn[i] + carry;
        carry = (limb)(p >> 64);
        dlimb t = (dlimb)un[i + j] - (limb)p - borrow;
        un[i + j] = (limb)t;
        borrow = (limb)((t >> 64) & 1U);
      }
      dlimb t = (dlimb)un[j + n] - carry - borrow;
      un[j + n] = (limb)t;
      bool negative = (t >> 64) & 1U;
      if (negative) {
        --qhat;
        limb c = 0;
        for (unsigned i = 0; i < n; ++i) {
          dlimb s2 = (dlimb)un[i + j] + vn[i] + c;
          un[i + j] = (limb)s2; c = (limb)(s2 >> 64);
        }
        un[j + n] += c;
      }
      qd[j] = (limb)qhat;
    }
    qq.neg_ = false; qq.trim();
    cpp_int rr; rr.reserve(n); rr.size_ = n;
    limb* rd = rr.data();
    for (unsigned i = 0; i < n; ++i)
      rd[i] = s ? (un[i] >> s) | (un[i + 1] << (64 - s)) : un[i];
    rr.neg_ = false; rr.trim();
    if (heap) { delete[] vn; delete[] un; }
    q = std::move(qq); r = std::move(rr);
  }
  void shl(unsigned long long s) {
    if (size_ == 0 || s == 0) return;
    unsigned ls = (unsigned)(s / 64), bs = (unsigned)(s % 64);
    unsigned n = size_ + ls + 1;
    reserve(n);
    limb* d = data();
    for (unsigned i = size_; i < n; ++i) d[i] = 0;
    for (unsigned i = n; i-- > 0;) {
      limb hi = (i >= ls && i - ls < size_) ? d[i - ls] : 0;
      limb lo = (i >= ls + 1 && i - ls - 1 < size_) ? d[i - ls - 1] : 0;
      d[i] = bs ? (hi << bs) | (lo >> (64 - bs)) : hi;
    }
    size_ = n;
    bool n0 = neg_; trim(); if (size_) neg_ = n0;
  }
  // arithmetic right shift (floor), as for two's complement values
  void shr(unsigned long long s) {
    if (size_ == 0 || s == 0) return;
    bool inexact = false;
    if (neg_) {
      for (unsigned long long i = 0; i < s && i < (unsigned long long)size_ * 64; ++i)
        if (test_bit(i)) { inexact = true; break; }
    }
    unsigned ls = (unsigned)std::min<unsigned long long>(s / 64, size_), bs = (unsigned)(s % 64);
    limb* d = data();
    unsigned n = size_ - ls;
    for (unsigned i = 0; i < n; ++i) {
      limb lo = d[i + ls];
      limb hi = (i + ls + 1 < size_) ? d[i + ls + 1] : 0;
      d[i] = bs ? (lo >> bs) | (hi << (64 - bs)) : lo;
    }
    size_ = n;
    bool n0 = neg_; trim(); if (size_) neg_ = n0;
    if (n0 && inexact) { neg_ = false; add_mag_one(); neg_ = true; }
  }
  void add_mag_one() { limb one = 1; add_mag(&one, 1); }
  void bitop(const cpp_int& b, int kind) {
    if (neg_ || b.neg_) throw std::domain_error("bitwise operations on negative values are not supported");
    unsigned n = std::max(size_, b.size_);
    reserve(n);
    limb* d = data();
    for (unsigned i = size_; i < n; ++i) d[i] = 0;
    const limb* bd = b.data();
    for (unsigned i = 0; i < n; ++i) {
      limb bi = i < b.size_ ? bd[i] : 0;
      d[i] = kind == 0 ? (d[i] & bi) : kind == 1 ? (d[i] | bi) : (d[i] ^ bi);
    }
    size_ = n; trim();
  }
};

using int128_t = cpp_int;
using int256_t = cpp_int;
using uint128_t = cpp_int;

inline unsigned long long msb(const cpp_int& v) { return v.msb_index(); }
inline unsigned long long lsb(const cpp_int& v) { return v.lsb_index(); }
inline bool bit_test(const cpp_int& v, unsigned long long i) { return v.test_bit(i); }
inline void divide_qr(const cpp_int& a, const cpp_int& b, cpp_int& q, cpp_int& r) { cpp_int::divmod(a, b, q, r); }
inline cpp_int abs(const cpp_int& v) { return v < 0 ? -v : v; }

}  // namespace multiprecision
}  // namespace boost
