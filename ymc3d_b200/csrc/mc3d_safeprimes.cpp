/*
 * mc3d_safeprimes.cpp -- multipliers for the multiply-with-carry generator.
 *
 * The reference seeds its generators from safeprimes_base32.txt
 * (src/mc3d_rng.cu:16, gpumcml_rng/gpumcml_rng.cu:72-97), a file it does not
 * distribute.  For base b = 2^32 a multiplier a gives a full-period MWC generator
 * when p = a b - 1 and (p - 1)/2 = a 2^31 - 1 are both prime (Marsaglia's
 * condition; the period is then (p - 1)/2).  This file enumerates such a in
 * descending order below a bound: a segmented sieve over a removes candidates
 * with a small prime factor in either number, and the survivors go through a
 * deterministic Miller-Rabin test for 64-bit integers (bases 2, 325, 9375, 28178,
 * 450775, 9780504, 1795265022, which decide every n < 2^64).
 */
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/mc3d.h"

namespace {

typedef unsigned __int128 u128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)((u128)a * b % m); }

uint64_t powmod(uint64_t a, uint64_t e, uint64_t m)
{
    uint64_t r = 1 % m;
    a %= m;
    while (e) {
        if (e & 1) r = mulmod(r, a, m);
        a = mulmod(a, a, m);
        e >>= 1;
    }
    return r;
}

bool is_prime_u64(uint64_t n)
{
    if (n < 2) return false;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t p : small) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    uint64_t d = n - 1;
    int r = 0;
    while ((d & 1) == 0) {
        d >>= 1;
        r++;
    }
    static const uint64_t bases[] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    for (uint64_t b : bases) {
        uint64_t a = b % n;
        if (a == 0) continue;
        uint64_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int i = 1; i < r; i++) {
            x = mulmod(x, x, n);
            if (x == n - 1) {
                comp = false;
                break;
            }
        }
        if (comp) return false;
    }
    return true;
}

struct Sieve {
    std::vector<uint32_t> primes; /* odd primes below 2^16 */
    std::vector<uint32_t> root32; /* a with a 2^32 = 1 mod q */
    std::vector<uint32_t> root31; /* a with a 2^31 = 1 mod q */
    Sieve()
    {
        const uint32_t lim = 1u << 16;
        std::vector<char> comp(lim, 0);
        for (uint32_t i = 3; i < lim; i += 2) {
            if (comp[i]) continue;
            primes.push_back(i);
            for (uint64_t j = (uint64_t)i * i; j < lim; j += 2 * i) comp[j] = 1;
        }
        for (uint32_t q : primes) {
            uint64_t t32 = ((uint64_t)1 << 32) % q, t31 = ((uint64_t)1 << 31) % q;
            root32.push_back((uint32_t)powmod(t32, q - 2, q)); /* inverse mod prime q */
            root31.push_back((uint32_t)powmod(t31, q - 2, q));
        }
    }
};

/* qualifying multipliers in [lo, hi), descending */
void segment(const Sieve &sv, uint64_t lo, uint64_t hi, std::vector<uint32_t> &out)
{
    size_t len = (size_t)(hi - lo);
    std::vector<char> bad(len, 0);
    for (size_t t = 0; t < sv.primes.size(); t++) {
        uint64_t q = sv.primes[t];
        for (uint64_t root : {(uint64_t)sv.root32[t], (uint64_t)sv.root31[t]}) {
            uint64_t start = lo + ((root + q - lo % q) % q);
            for (uint64_t a = start; a < hi; a += q) bad[a - lo] = 1;
        }
    }
    for (size_t k = len; k-- > 0;) {
        if (bad[k]) continue;
        uint64_t a = lo + k;
        if (a < 2) continue;
        if (!is_prime_u64((a << 31) - 1)) continue;
        if (!is_prime_u64((a << 32) - 1)) continue;
        out.push_back((uint32_t)a);
    }
}

} /* namespace */

extern "C" {

int mc3d_safeprime_table(uint32_t *out, int64_t n, uint64_t below, int32_t threads)
{
    if (!out || n < 0) return MC3D_ERR_ARG;
    if (below == 0 || below > (1ull << 32)) below = 1ull << 32;
    if (threads <= 0) threads = (int32_t)std::max(1u, std::thread::hardware_concurrency());
    static const Sieve sv;
    const uint64_t seg = 1u << 20;
    int64_t have = 0;
    uint64_t top = below;
    while (have < n && top > 2) {
        int nt = threads;
        std::vector<std::vector<uint32_t>> parts(nt);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; t++) {
            uint64_t hi = top > (uint64_t)t * seg ? top - (uint64_t)t * seg : 0;
            uint64_t lo = hi > seg ? hi - seg : 2;
            if (hi <= lo) continue;
            pool.emplace_back([&, t, lo, hi] { segment(sv, lo, hi, parts[t]); });
        }
        for (auto &th : pool) th.join();
        for (int t = 0; t < nt && have < n; t++)
            for (uint32_t a : parts[t]) {
                if (have >= n) break;
                out[have++] = a;
            }
        top = top > (uint64_t)nt * seg ? top - (uint64_t)nt * seg : 2;
    }
    return have == n ? MC3D_OK : MC3D_ERR_TABLE;
}

int mc3d_safeprimes_write(const char *path, const uint32_t *table, int64_t n)
{
    if (!path || (!table && n > 0)) return MC3D_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return MC3D_ERR_IO;
    for (int64_t i = 0; i < n; i++) {
        uint64_t p = ((uint64_t)table[i] << 32) - 1;
        fprintf(f, "%u %u %u\n", table[i], (uint32_t)(p >> 32), (uint32_t)p);
    }
    int bad = ferror(f);
    if (fclose(f) != 0 || bad) return MC3D_ERR_IO;
    return MC3D_OK;
}

int mc3d_safeprimes_read(const char *path, uint32_t *out, int64_t cap, int64_t *n_read)
{
    if (!path || !out || cap < 0) return MC3D_ERR_ARG;
    if (n_read) *n_read = 0;
    FILE *f = fopen(path, "r");
    if (!f) return MC3D_ERR_IO;
    int64_t n = 0;
    unsigned a, t1, t2;
    while (n < cap && fscanf(f, "%u %u %u", &a, &t1, &t2) == 3) out[n++] = a;
    fclose(f);
    if (n_read) *n_read = n;
    return n > 0 ? MC3D_OK : MC3D_ERR_FORMAT;
}

} /* extern "C" */
