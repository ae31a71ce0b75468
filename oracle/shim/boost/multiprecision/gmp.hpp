/* Minimal stand-in for boost::multiprecision::{mpz_int, mpf_float}.  The reference
 * uses them only in its string codecs; the integer codec path never touches them.
 * mpz_int is a thin __int128 wrapper with the operators that bit_write.h's string
 * writer names, so that header compiles. */
#pragma once
#include <gmp.h>
namespace boost { namespace multiprecision {
struct mpz_int {
  __int128 v = 0;
  mpz_int() = default;
  template <class X> mpz_int(X x) : v((__int128)x) {}
  template <class X> X convert_to() const { return (X)v; }
  friend mpz_int operator&(mpz_int a, mpz_int b) { mpz_int r; r.v = a.v & b.v; return r; }
  friend mpz_int operator|(mpz_int a, mpz_int b) { mpz_int r; r.v = a.v | b.v; return r; }
  friend mpz_int operator+(mpz_int a, mpz_int b) { mpz_int r; r.v = a.v + b.v; return r; }
  friend mpz_int operator-(mpz_int a, mpz_int b) { mpz_int r; r.v = a.v - b.v; return r; }
  friend mpz_int operator*(mpz_int a, mpz_int b) { mpz_int r; r.v = a.v * b.v; return r; }
  mpz_int operator-() const { mpz_int r; r.v = -v; return r; }
  template <class S> mpz_int operator<<(S s) const { mpz_int r; r.v = v << s; return r; }
  template <class S> mpz_int operator>>(S s) const { mpz_int r; r.v = v >> s; return r; }
  mpz_int &operator+=(mpz_int b) { v += b.v; return *this; }
  mpz_int &operator-=(mpz_int b) { v -= b.v; return *this; }
  friend bool operator<(mpz_int a, mpz_int b) { return a.v < b.v; }
  friend bool operator>(mpz_int a, mpz_int b) { return a.v > b.v; }
  friend bool operator<=(mpz_int a, mpz_int b) { return a.v <= b.v; }
  friend bool operator>=(mpz_int a, mpz_int b) { return a.v >= b.v; }
  friend bool operator==(mpz_int a, mpz_int b) { return a.v == b.v; }
  friend bool operator!=(mpz_int a, mpz_int b) { return a.v != b.v; }
};
struct mpf_float { double v = 0; mpf_float() = default; template <class X> mpf_float(X x) : v((double)x) {} };
}}
