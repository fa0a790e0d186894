/* Minimal gmpxx stand-in (see gmp.h in this folder): an mpz_class over a
 * signed 128-bit integer with the members the reference's Goldilocks headers
 * call (goldilocks_base_field_tools.hpp:72-186): construction from integers
 * and strings, + - * / %, comparisons, get_ui/get_si/get_str, get_mpz_t.
 * Test infrastructure only (backs the reference CPU build under oracle/_ref).
 */
#ifndef ORACLE_SHIM_GMPXX_H
#define ORACLE_SHIM_GMPXX_H

/* the real gmpxx.h brings these in; the reference sources rely on it */
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>

#include "gmp.h"

class mpz_class
{
    mpz_t z;

public:
    mpz_class() { z->v = 0; }
    mpz_class(int a) { z->v = a; }
    mpz_class(long a) { z->v = a; }
    mpz_class(long long a) { z->v = a; }
    mpz_class(unsigned int a) { z->v = a; }
    mpz_class(unsigned long a) { z->v = (__int128)a; }
    mpz_class(unsigned long long a) { z->v = (__int128)a; }
    mpz_class(const std::string &s, int radix = 10) { z->v = parse(s, radix); }
    mpz_class(const char *s, int radix = 10) { z->v = parse(std::string(s), radix); }
    mpz_class(const mpz_class &o) { z->v = o.z->v; }
    mpz_class &operator=(const mpz_class &o)
    {
        z->v = o.z->v;
        return *this;
    }

    static __int128 parse(const std::string &s, int radix)
    {
        size_t i = 0;
        bool neg = false;
        if (i < s.size() && (s[i] == '-' || s[i] == '+')) {
            neg = s[i] == '-';
            i++;
        }
        if (radix == 0) {
            radix = 10;
            if (s.size() > i + 1 && s[i] == '0' && (s[i + 1] == 'x' || s[i + 1] == 'X')) {
                radix = 16;
                i += 2;
            }
        } else if (radix == 16 && s.size() > i + 1 && s[i] == '0' && (s[i + 1] == 'x' || s[i + 1] == 'X')) {
            i += 2;
        }
        __int128 v = 0;
        for (; i < s.size(); i++) {
            char c = s[i];
            int d;
            if (c >= '0' && c <= '9') d = c - '0';
            else if (c >= 'a' && c <= 'z') d = c - 'a' + 10;
            else if (c >= 'A' && c <= 'Z') d = c - 'A' + 10;
            else throw std::invalid_argument("mpz_class: bad digit");
            if (d >= radix) throw std::invalid_argument("mpz_class: bad digit");
            v = v * radix + d;
        }
        return neg ? -v : v;
    }

    mpz_ptr get_mpz_t() { return z; }
    mpz_srcptr get_mpz_t() const { return z; }
    unsigned long get_ui() const { return mpz_get_ui(z); }
    long get_si() const { return mpz_get_si(z); }
    std::string get_str(int radix = 10) const
    {
        static const char digits[] = "0123456789abcdefghijklmnopqrstuvwxyz";
        __int128 v = z->v;
        bool neg = v < 0;
        unsigned __int128 u = neg ? (unsigned __int128)(-v) : (unsigned __int128)v;
        if (u == 0) return "0";
        std::string out;
        while (u) {
            out.insert(out.begin(), digits[(int)(u % (unsigned)radix)]);
            u /= (unsigned)radix;
        }
        if (neg) out.insert(out.begin(), '-');
        return out;
    }

    friend mpz_class operator+(const mpz_class &a, const mpz_class &b) { return mk(a.z->v + b.z->v); }
    friend mpz_class operator-(const mpz_class &a, const mpz_class &b) { return mk(a.z->v - b.z->v); }
    friend mpz_class operator*(const mpz_class &a, const mpz_class &b) { return mk(a.z->v * b.z->v); }
    /* GMP's operator/ and operator% truncate toward zero, as C does */
    friend mpz_class operator/(const mpz_class &a, const mpz_class &b) { return mk(a.z->v / b.z->v); }
    friend mpz_class operator%(const mpz_class &a, const mpz_class &b) { return mk(a.z->v % b.z->v); }
    friend bool operator<(const mpz_class &a, const mpz_class &b) { return a.z->v < b.z->v; }
    friend bool operator>(const mpz_class &a, const mpz_class &b) { return a.z->v > b.z->v; }
    friend bool operator<=(const mpz_class &a, const mpz_class &b) { return a.z->v <= b.z->v; }
    friend bool operator>=(const mpz_class &a, const mpz_class &b) { return a.z->v >= b.z->v; }
    friend bool operator==(const mpz_class &a, const mpz_class &b) { return a.z->v == b.z->v; }
    friend bool operator!=(const mpz_class &a, const mpz_class &b) { return a.z->v != b.z->v; }

private:
    static mpz_class mk(__int128 v)
    {
        mpz_class r;
        r.z->v = v;
        return r;
    }
};

#endif
