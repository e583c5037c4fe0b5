/*
 * Noise injection for running the reference's own code deterministically
 * (oracle test infrastructure only).
 *
 * The reference draws every Gaussian from a thread-local std::ranlux24 seeded
 * with clock() + hash(thread id) (field.h:692-696, 2131-2135, 2262-2266), so no
 * two runs agree.  To feed it the same noise the device engine uses, this
 * header is included BEFORE the reference's headers and replaces, by macro,
 * the two std names those functions use:
 *     std::ranlux24                  -> std::jw_injected_engine (seed ignored)
 *     std::normal_distribution<T>    -> std::jw_injected_normal<T>
 * The replacement distribution returns  z * stddev + mean,  the same expression
 * libstdc++'s normal_distribution applies to its unit normal, with z taken in
 * order from an injected stream.  The reference's loops must then run
 * serially (build WITHOUT -fopenmp) so that the draw order is the source
 * order: per site i, n[0..7] (setMVModel, field.h:703-705) or
 * n[0], m[0], n[1], m[1], ... (generate_gaussian, field.h:2170-2173).
 *
 * The stream is either a memory buffer (jw_inject_set) or, when the
 * environment variable JW_INJECT_FILE names a file of native doubles, that
 * file (loaded on the first draw).  Running past the end aborts loudly.
 */
#ifndef JW_ORACLE_INJECT_H
#define JW_ORACLE_INJECT_H

#include <random>
#include <stdio.h>
#include <stdlib.h>

struct jw_inject_state {
    const double* z = nullptr;
    long n = 0;
    long pos = 0;
    double* owned = nullptr;
};

inline jw_inject_state& jw_inject_global() {
    static jw_inject_state s;
    return s;
}

inline void jw_inject_set(const double* z, long n) {
    jw_inject_state& s = jw_inject_global();
    s.z = z;
    s.n = n;
    s.pos = 0;
}

inline double jw_inject_next() {
    jw_inject_state& s = jw_inject_global();
    if (!s.z) {
        const char* path = getenv("JW_INJECT_FILE");
        if (path) {
            FILE* f = fopen(path, "rb");
            if (!f) { fprintf(stderr, "inject: cannot open %s\n", path); abort(); }
            fseek(f, 0, SEEK_END);
            long bytes = ftell(f);
            fseek(f, 0, SEEK_SET);
            s.owned = (double*)malloc((size_t)bytes);
            if (fread(s.owned, 1, (size_t)bytes, f) != (size_t)bytes) { fprintf(stderr, "inject: short read\n"); abort(); }
            fclose(f);
            s.z = s.owned;
            s.n = bytes / (long)sizeof(double);
            s.pos = 0;
        }
    }
    if (!s.z || s.pos >= s.n) {
        fprintf(stderr, "inject: noise stream exhausted after %ld draws\n", s.pos);
        abort();
    }
    return s.z[s.pos++];
}

namespace std {
struct jw_injected_engine {
    template <class S>
    explicit jw_injected_engine(S) {}
};
template <class R>
struct jw_injected_normal {
    R mean_, stddev_;
    jw_injected_normal(R mean, R stddev) : mean_(mean), stddev_(stddev) {}
    template <class G>
    R operator()(G&) { return (R)jw_inject_next() * stddev_ + mean_; }
};
}  // namespace std

#define ranlux24 jw_injected_engine
#define normal_distribution jw_injected_normal

#endif
