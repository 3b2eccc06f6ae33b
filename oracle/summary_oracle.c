/*
 * summary_oracle.c -- TEST INFRASTRUCTURE (oracle).  Plain-C restatement of the
 * sequence pass of AnchorWave's alignment selector: summarizeSequencePair
 * (src/myImportandFunction/AlignmentAlgorithmSelector.cpp:730-757) over
 * SequenceProfileAccumulator (:591-728), with mixHash (:561-568), encodedBase
 * (:581-589), the constants of :28-34 and the sampling modulos of
 * makeAlignmentSelectionPlan (:1752-1760).  Used only by tests/ and the CPU leg of
 * bench.py to check the CUDA summary; pinned against the compiled selector
 * (oracle/_ref, ref_selector_shim.cpp).
 *
 * Per sequence: FNV-1a fingerprint of the bytes finished by mixHash with the length,
 * ambiguous fraction (bases other than A/C/G/T in any case), low-complexity fraction
 * (bases at run length >= 4 of one base), normalized entropy (per 64-base block:
 * Shannon entropy of the valid bases / 2 x valid bases, summed and divided by the
 * length), and three strand-aware k-mer sketches (k = 9, 15, 21): the k-mers of
 * valid bases whose mixHash is divisible by the scale's modulo, in position order, at
 * most 4 entries per hash value.
 */
#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const uint64_t os_k[3] = {9, 15, 21};
static const uint64_t os_target[3] = {1024, 4096, 1024};
#define OS_BLOCK 64
#define OS_MAX_OCC 4

typedef struct {
    uint64_t fingerprint;
    double ambiguous_fraction, normalized_entropy, low_complexity_fraction;
    int64_t count[3];
} os_summary;

static uint64_t os_mix(uint64_t v) {
    v ^= v >> 30;
    v *= 0xbf58476d1ce4e5b9ULL;
    v ^= v >> 27;
    v *= 0x94d049bb133111ebULL;
    v ^= v >> 31;
    return v;
}

static int os_code(char b) {
    switch (toupper((unsigned char)b)) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    default: return -1;
    }
}

/* occurrences per hash value: open addressing, grown at half load */
typedef struct {
    uint64_t *key;
    uint8_t *cnt, *used;
    size_t cap, n;
} os_map;
static uint8_t *os_slot(os_map *m, uint64_t h) {
    if (2 * (m->n + 1) > m->cap) {
        os_map g = {0, 0, 0, m->cap ? 2 * m->cap : 1024, 0};
        g.key = (uint64_t *)calloc(g.cap, 8), g.cnt = (uint8_t *)calloc(g.cap, 1), g.used = (uint8_t *)calloc(g.cap, 1);
        for (size_t i = 0; i < m->cap; ++i)
            if (m->used[i]) *os_slot(&g, m->key[i]) = m->cnt[i];
        free(m->key), free(m->cnt), free(m->used);
        *m = g;
    }
    size_t i = (size_t)(os_mix(h) & (m->cap - 1));
    while (m->used[i] && m->key[i] != h) i = (i + 1) & (m->cap - 1);
    if (!m->used[i]) m->used[i] = 1, m->key[i] = h, m->cnt[i] = 0, ++m->n;
    return &m->cnt[i];
}

/* One sequence (SequenceProfileAccumulator::consume over every base, then finish).
 * Sketch entries go to hash/pos from *w on (room permitting); counts always. */
static void os_sequence(const char *s, int64_t len, const uint64_t *mod, os_summary *o, uint64_t *hash, uint32_t *pos,
                        int64_t cap, int64_t *w) {
    uint64_t fp = 1469598103934665603ULL, amb = 0, tail = 0, run = 0, bb = 0, cnt[5] = {0, 0, 0, 0, 0};
    uint64_t roll[3] = {0, 0, 0}, valid[3] = {0, 0, 0};
    long double weighted = 0.0L;
    int prev = -1;
    os_map occ[3];
    memset(occ, 0, sizeof(occ));
    for (int sc = 0; sc < 3; ++sc) o->count[sc] = 0;
    /* entries of scale sc are buffered so that the output is grouped by scale */
    uint64_t *eh[3];
    uint32_t *ep[3];
    int64_t en[3] = {0, 0, 0}, ec[3] = {256, 256, 256};
    for (int sc = 0; sc < 3; ++sc) eh[sc] = (uint64_t *)malloc(8 * 256), ep[sc] = (uint32_t *)malloc(4 * 256);
    for (int64_t p = 0; p <= len; ++p) {
        if (p == len || bb == OS_BLOCK) { /* finishEntropyBlock */
            if (bb) {
                const uint64_t vb = bb - cnt[4];
                long double ent = 0.0L;
                if (vb) {
                    for (int b = 0; b < 4; ++b) {
                        if (!cnt[b]) continue;
                        const long double pr = (long double)cnt[b] / (long double)vb;
                        ent -= pr * log2l(pr);
                    }
                    ent = ent / 2.0L * (long double)vb / (long double)bb;
                }
                weighted += ent * (long double)bb;
                memset(cnt, 0, sizeof(cnt));
                bb = 0;
            }
            if (p == len) break;
        }
        const unsigned char raw = (unsigned char)s[p];
        fp ^= (uint64_t)raw;
        fp *= 1099511628211ULL;
        const int c = os_code(s[p]);
        if (c < 0) {
            ++amb, prev = -1, run = 0, cnt[4] += 1;
            for (int sc = 0; sc < 3; ++sc) roll[sc] = 0, valid[sc] = 0;
        } else {
            if (c == prev) ++run;
            else prev = c, run = 1;
            if (run >= 4) ++tail;
            cnt[c] += 1;
            for (int sc = 0; sc < 3; ++sc) {
                const uint64_t k = os_k[sc], mask = (1ULL << (2 * k)) - 1;
                roll[sc] = ((roll[sc] << 2) | (uint64_t)c) & mask;
                if (++valid[sc] < k) continue;
                const uint64_t h = os_mix(roll[sc]);
                if (h % mod[sc] != 0) continue;
                uint8_t *oc = os_slot(&occ[sc], h);
                if (*oc >= OS_MAX_OCC) continue;
                ++*oc;
                if (en[sc] == ec[sc]) {
                    ec[sc] *= 2;
                    eh[sc] = (uint64_t *)realloc(eh[sc], 8 * (size_t)ec[sc]);
                    ep[sc] = (uint32_t *)realloc(ep[sc], 4 * (size_t)ec[sc]);
                }
                eh[sc][en[sc]] = h, ep[sc][en[sc]] = (uint32_t)((uint64_t)p + 1 - k), ++en[sc];
            }
        }
        ++bb;
    }
    for (int sc = 0; sc < 3; ++sc) {
        o->count[sc] = en[sc];
        for (int64_t i = 0; i < en[sc]; ++i, ++*w)
            if (*w < cap) hash[*w] = eh[sc][i], pos[*w] = ep[sc][i];
        free(eh[sc]), free(ep[sc]);
        free(occ[sc].key), free(occ[sc].cnt), free(occ[sc].used);
    }
    o->fingerprint = os_mix(fp ^ os_mix((uint64_t)len));
    o->ambiguous_fraction = o->low_complexity_fraction = o->normalized_entropy = 0.0;
    if (len) {
        o->ambiguous_fraction = (double)amb / (double)len;
        o->low_complexity_fraction = (double)tail / (double)len;
        o->normalized_entropy = (double)(weighted / (long double)len);
    }
}

/* The sampling modulos of makeAlignmentSelectionPlan for a pair. */
void oracle_summary_modulos(int64_t qlen, int64_t rlen, uint64_t *mod) {
    const uint64_t mx = (uint64_t)(qlen > rlen ? qlen : rlen);
    for (int sc = 0; sc < 3; ++sc) {
        const uint64_t avail = mx >= os_k[sc] ? mx - os_k[sc] + 1 : 0;
        mod[sc] = avail / os_target[sc] > 1 ? avail / os_target[sc] : 1;
    }
}

/* summarizeSequencePair(query, reference, modulos, identical).  modulos NULL: those of
 * makeAlignmentSelectionPlan.  out[0] query, out[1] reference; sketch entries back to
 * back (query k=9, 15, 21, then reference); returns the number of entries (written only
 * up to cap). */
int64_t oracle_sequence_summary(const char *query, int64_t qlen, const char *reference, int64_t rlen,
                                const uint64_t *modulos, os_summary *out, int *identical, uint64_t *hash,
                                uint32_t *pos, int64_t cap) {
    uint64_t mod[3];
    if (modulos) memcpy(mod, modulos, sizeof(mod));
    else oracle_summary_modulos(qlen, rlen, mod);
    *identical = qlen == rlen && (qlen == 0 || memcmp(query, reference, (size_t)qlen) == 0);
    int64_t w = 0;
    os_sequence(query, qlen, mod, &out[0], hash, pos, cap, &w);
    os_sequence(reference, rlen, mod, &out[1], hash, pos, cap, &w);
    return w;
}

int oracle_sizeof_summary(void) { return (int)sizeof(os_summary); }
