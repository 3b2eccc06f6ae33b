// AnchorWave's two rescue procedures for intervals that the exact engines cannot take,
// batched over many intervals on the GPU KSW2 kernels (host orchestration; every DP pass is
// one aw_ksw_extd2_batch call per scoring flag):
//   * alignScoreCertifiedKsw2 (src/myImportandFunction/alignSlidingWindow.cpp:1197-1400): the
//     unbanded score-only optimum, then banded tracebacks at growing bands until the
//     re-scored alignment reaches that optimum, the skipped smallest band only on failure;
//   * alignSlidingWindow (:457-590): one global alignment when the interval fits the window
//     envelope, else semiglobal windows of W+1 bases advancing to the better end.
// Round k of a batch runs the k-th DP of every interval still in progress, so each interval
// gets exactly the result a call of its own would give.  The selector's chained traceback
// (a selection plan, :1256-1289) stays with the caller.
#include "aw_internal.h"
#include "../../include/anchorwave_b200.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

constexpr int kCompleted = 0, kTimeLimit = 1, kNotCertified = 2, kFailed = 3;  // Ksw2CertifiedStatus
// band cells an interval's run-ahead round may take (several narrow bands of a long interval)
constexpr double kAheadCells = 4e9;

// encodeKswSequence (alignSlidingWindow.cpp:645-660)
int encode(const std::string &s, std::vector<uint8_t> &out) {
    int flag = 0;
    out.resize(s.size());
    for (size_t i = 0; i < s.size(); ++i) {
        switch (s[i]) {
        case 'A': case 'a': out[i] = 0; break;
        case 'C': case 'c': out[i] = 1; break;
        case 'G': case 'g': out[i] = 2; break;
        case 'T': case 't': out[i] = 3; break;
        default: out[i] = 4, flag = AW_EZ_GENERIC_SC;
        }
    }
    return flag;
}

// gappedAlignmentReconstructs (:662-675)
bool reconstructs(const std::string &aln, const std::string &seq) {
    size_t p = 0;
    for (char b : aln) {
        if (b == '-') continue;
        if (p >= seq.size() || seq[p] != b) return false;
        ++p;
    }
    return p == seq.size();
}

// scoreGappedTwoPieceAffineAlignment (:677-721); penalties negative.  Throws like the
// reference on rows of different lengths or a column with two gaps.
int64_t rescore(const std::string &q, const std::string &d, int mis, int o1, int e1, int o2, int e2) {
    if (q.size() != d.size()) throw std::runtime_error("KSW2 returned alignment rows with different lengths");
    int64_t s = 0;
    size_t c = 0;
    while (c < q.size()) {
        const bool qg = q[c] == '-', dg = d[c] == '-';
        if (qg && dg) throw std::runtime_error("KSW2 returned an alignment column with two gaps");
        if (qg || dg) {
            size_t e = c + 1;
            while (e < q.size() && (q[e] == '-') == qg && (d[e] == '-') != qg) ++e;
            const int64_t L = (int64_t)(e - c);
            s += std::max<int64_t>((int64_t)o1 + (int64_t)e1 * L, (int64_t)o2 + (int64_t)e2 * L);
            c = e;
            continue;
        }
        if (q[c] != d[c]) s += mis;
        ++c;
    }
    return s;
}

// The CIGAR -> gapped rows decoding of :307-324 / :855-870 (M, = and X copy both, I the
// query, D the reference).  Returns the bases consumed of each sequence.
void rows(const ksw_extz_t &ez, const std::string &q, const std::string &d, std::string &aq, std::string &ad,
          int64_t &qp, int64_t &tp) {
    aq.clear(), ad.clear(), qp = 0, tp = 0;
    for (int i = 0; i < ez.n_cigar; ++i) {
        const int64_t L = ez.cigar[i] >> 4;
        const int op = ez.cigar[i] & 0xf;
        if (op == 0 || op == 7 || op == 8) {
            aq.append(q, (size_t)qp, (size_t)L), ad.append(d, (size_t)tp, (size_t)L);
            qp += L, tp += L;
        } else if (op == 1) {
            aq.append(q, (size_t)qp, (size_t)L), ad.append((size_t)L, '-');
            qp += L;
        } else if (op == 2) {
            aq.append((size_t)L, '-'), ad.append(d, (size_t)tp, (size_t)L);
            tp += L;
        }
    }
}

std::vector<int8_t> matrix(int mis) {
    const int8_t b = (int8_t)(mis < 0 ? mis : -mis);
    std::vector<int8_t> m(25);
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) m[i * 5 + j] = i == j ? 0 : b;
    return m;
}

struct Job {
    int id;
    std::string q, d;  // the sequences of this DP (a window, or the whole interval)
    int band;          // -1: full
};

// One DP round: the jobs grouped by scoring flag (GENERIC_SC when a base is not ACGT), one
// batched call per group.  Results are indexed like `jobs`; the caller frees their CIGARs.
int run_round(const std::vector<Job> &jobs, int mis, int o1, int e1, int o2, int e2, int flag_extra,
              std::vector<ksw_extz_t> &res) {
    res.assign(jobs.size(), ksw_extz_t{});
    std::vector<std::vector<uint8_t>> qc(jobs.size()), tc(jobs.size());
    std::map<int, std::vector<size_t>> groups;
    for (size_t k = 0; k < jobs.size(); ++k) {
        const int f = encode(jobs[k].q, qc[k]) | encode(jobs[k].d, tc[k]);
        groups[f].push_back(k);
    }
    const std::vector<int8_t> mat = matrix(mis);
    for (auto &g : groups) {
        const std::vector<size_t> &ks = g.second;
        const int n = (int)ks.size();
        std::vector<int> ql(n), tl(n), w(n);
        std::vector<const uint8_t *> qp(n), tp(n);
        std::vector<ksw_extz_t> ez(n);
        for (int a = 0; a < n; ++a) {
            const size_t k = ks[a];
            ql[a] = (int)qc[k].size(), tl[a] = (int)tc[k].size(), w[a] = jobs[k].band;
            qp[a] = qc[k].data(), tp[a] = tc[k].data();
            memset(&ez[a], 0, sizeof(ksw_extz_t));
        }
        const int rc = aw_ksw_extd2_batch(n, ql.data(), qp.data(), tl.data(), tp.data(), w.data(), 5, mat.data(),
                                          (int8_t)-o1, (int8_t)-e1, (int8_t)-o2, (int8_t)-e2, -1, 0,
                                          g.first | flag_extra, ez.data());
        for (int a = 0; a < n; ++a) res[ks[a]] = ez[a];
        if (rc != AW_OK) return rc;
    }
    return AW_OK;
}

char *dup(const std::string &s) {
    char *p = (char *)malloc(s.size() + 1);
    if (!p) return nullptr;
    memcpy(p, s.data(), s.size());
    p[s.size()] = 0;
    return p;
}

struct Cert {
    int status = kFailed;
    int64_t score = 0, optimal = 0, final_band = -1, attempts = 0;
    std::string aq, ad, bq, bd;
    // band schedule (:1296-1347) and the failure-only smallest band (:1351-1352)
    std::vector<int64_t> bands;
    int64_t fallback = -1, last_band = 0;
    bool active = false, done = false;
};

// Folds one banded traceback into the procedure's state (:1316-1340 / :1364-1393).
void take_band(Cert &r, const ksw_extz_t &ez, const std::string &q, const std::string &d, int64_t band, int mis,
               int o1, int e1, int o2, int e2) {
    ++r.attempts;
    if (ez.stopped) {
        r.status = kTimeLimit, r.done = true;
        return;
    }
    std::string aq, ad;
    int64_t qp, tp;
    rows(ez, q, d, aq, ad, qp, tp);
    const int64_t s = rescore(aq, ad, mis, o1, e1, o2, e2);
    const bool valid = aq.size() == ad.size() && reconstructs(aq, q) && reconstructs(ad, d);
    if (s == r.optimal && valid) {
        r.score = s, r.final_band = band, r.aq = std::move(aq), r.ad = std::move(ad);
        r.status = kCompleted, r.done = true;
    } else if (valid && (r.bq.empty() || s > r.score)) {
        r.score = s, r.bq = std::move(aq), r.bd = std::move(ad);
    }
}

void free_ez(std::vector<ksw_extz_t> &v) {
    for (auto &z : v) free(z.cigar), z.cigar = nullptr;
}

}  // namespace

using namespace aw;

extern "C" {

int aw_align_score_certified_batch(int n, const char *const *query, const int64_t *qlen, const char *const *reference,
                                   const int64_t *rlen, const int64_t *initial_band_width,
                                   const int64_t *maximum_band_width, int32_t mis, int32_t o1, int32_t e1, int32_t o2,
                                   int32_t e2, double maximum_runtime_seconds,
                                   const int64_t *precomputed_optimal_scores, aw_certified_result_t *out) {
    if (n < 0 || (n > 0 && (!query || !qlen || !reference || !rlen || !out || !initial_band_width ||
                            !maximum_band_width)))
        return AW_E_INVAL;
    for (int i = 0; i < n; ++i)
        if (qlen[i] < 0 || rlen[i] < 0 || qlen[i] > INT32_MAX / 2 || rlen[i] > INT32_MAX / 2) return AW_E_INVAL;
    std::vector<Cert> C(n);
    std::vector<std::string> Q(n), D(n);
    std::vector<int> todo;
    for (int i = 0; i < n; ++i) {
        Q[i].assign(query[i] ? query[i] : "", (size_t)qlen[i]);
        D[i].assign(reference[i] ? reference[i] : "", (size_t)rlen[i]);
        Cert &r = C[i];
        const int64_t diff = std::llabs(qlen[i] - rlen[i]);
        if (std::min(qlen[i], rlen[i]) == 0) {
            // :1213-1229: the whole interval is one gap; ksw2ScoreOnly's gap score (:731-739)
            r.aq = Q[i].empty() ? std::string((size_t)rlen[i], '-') : Q[i];
            r.ad = D[i].empty() ? std::string((size_t)qlen[i], '-') : D[i];
            const int64_t L = std::max(qlen[i], rlen[i]);
            r.score = r.optimal = std::max<int64_t>((int64_t)o1 + (int64_t)e1 * L, (int64_t)o2 + (int64_t)e2 * L);
            r.final_band = 0, r.attempts = 1, r.status = kCompleted;
        } else if (initial_band_width[i] < 0 || maximum_band_width[i] < 0 || maximum_band_width[i] < diff) {
            r.status = kNotCertified;
        } else {
            todo.push_back(i);
        }
    }
    const bool timed = maximum_runtime_seconds > 0;
    if (timed) aw_ksw_set_deadline(maximum_runtime_seconds);
    int rc = AW_OK;
    try {
        if (precomputed_optimal_scores) {
            for (int i : todo) C[i].optimal = precomputed_optimal_scores[i];
        } else if (!todo.empty()) {
            std::vector<Job> jobs;
            for (int i : todo) jobs.push_back(Job{i, Q[i], D[i], -1});
            std::vector<ksw_extz_t> res;
            rc = run_round(jobs, mis, o1, e1, o2, e2, AW_EZ_SCORE_ONLY, res);
            for (size_t k = 0; k < jobs.size(); ++k) {
                Cert &r = C[jobs[k].id];
                r.optimal = res[k].score;
                if (res[k].stopped) r.status = kTimeLimit, r.done = true;
            }
            free_ez(res);
        }
        for (int i : todo) {
            Cert &r = C[i];
            if (r.done) continue;
            if (r.optimal == AW_NEG_INF) {
                r.status = kFailed, r.done = true;
                continue;
            }
            const int64_t diff = std::llabs(qlen[i] - rlen[i]);
            const int64_t max_band = std::min<int64_t>(std::max(qlen[i], rlen[i]), maximum_band_width[i]);
            const int64_t requested = std::max<int64_t>(diff, std::max<int64_t>(1, initial_band_width[i]));
            const int64_t doubled = requested * 2;
            int64_t band = std::min(max_band, std::max(requested, doubled));
            while (band >= diff && band <= max_band) {
                r.bands.push_back(band);
                if (band == max_band) break;
                const int64_t nxt = std::min(max_band, std::max(band + 1, band * 2));
                if (nxt <= band) break;
                band = nxt;
            }
            r.last_band = r.bands.empty() ? band : r.bands.back();
            r.fallback = requested < std::min(max_band, doubled) ? requested : -1;
            r.active = true;
        }
        // Untimed calls run ahead: a round takes an interval's next bands while their band
        // cells stay within kAheadCells together (always at least one band) and folds the
        // results in band order, dropping those after the certifying one, so every interval
        // ends in the state the band-by-band loop reaches.  A long interval at narrow bands is
        // bound by its strip chain, not by its cells, so the bands taken together cost about
        // one round.  Timed calls keep one band per round (the deadline then stops the same
        // attempts as the reference's loop would reach).
        std::vector<size_t> next(n, 0);
        while (rc == AW_OK) {
            std::vector<Job> jobs;
            for (int i : todo) {
                const Cert &r = C[i];
                if (!r.active || r.done) continue;
                double cells = 0.0;
                for (size_t b = next[i]; b < r.bands.size(); ++b) {
                    const double c = (double)std::max(qlen[i], rlen[i]) * (2.0 * (double)r.bands[b] + 1.0);
                    if (b > next[i] && (timed || cells + c > kAheadCells)) break;
                    cells += c;
                    jobs.push_back(Job{i, Q[i], D[i], (int)r.bands[b]});
                }
            }
            if (jobs.empty()) break;
            std::vector<ksw_extz_t> res;
            rc = run_round(jobs, mis, o1, e1, o2, e2, 0, res);
            if (rc == AW_OK)
                for (size_t k = 0; k < jobs.size(); ++k) {
                    const int i = jobs[k].id;
                    ++next[i];
                    if (!C[i].done) take_band(C[i], res[k], Q[i], D[i], jobs[k].band, mis, o1, e1, o2, e2);
                }
            free_ez(res);
        }
        if (rc == AW_OK) {
            std::vector<Job> jobs;
            for (int i : todo)
                if (C[i].active && !C[i].done && C[i].fallback >= 0) jobs.push_back(Job{i, Q[i], D[i], (int)C[i].fallback});
            if (!jobs.empty()) {
                std::vector<ksw_extz_t> res;
                rc = run_round(jobs, mis, o1, e1, o2, e2, 0, res);
                if (rc == AW_OK)
                    for (size_t k = 0; k < jobs.size(); ++k)
                        take_band(C[jobs[k].id], res[k], Q[jobs[k].id], D[jobs[k].id], jobs[k].band, mis, o1, e1, o2,
                                  e2);
                free_ez(res);
            }
        }
        for (int i : todo)
            if (C[i].active && !C[i].done) C[i].final_band = C[i].last_band, C[i].status = kNotCertified;
    } catch (const std::exception &ex) {
        set_error((std::string("aw_align_score_certified_batch: ") + ex.what()).c_str());
        rc = AW_E_INVAL;
    }
    if (timed) aw_ksw_set_deadline(0.0);
    for (int i = 0; i < n; ++i) {
        const Cert &r = C[i];
        aw_certified_result_t &o = out[i];
        memset(&o, 0, sizeof(o));
        o.status = r.status, o.score = r.score, o.optimal_score = r.optimal;
        o.final_band_width = r.final_band, o.traceback_attempts = r.attempts;
        if (r.status == kCompleted) {
            o.alignment_q = dup(r.aq), o.alignment_d = dup(r.ad), o.alignment_len = (int64_t)r.aq.size();
        }
        if (!r.bq.empty()) o.best_effort_q = dup(r.bq), o.best_effort_d = dup(r.bd), o.best_effort_len = (int64_t)r.bq.size();
    }
    return rc;
}

void aw_certified_result_free(aw_certified_result_t *r) {
    if (!r) return;
    free(r->alignment_q), free(r->alignment_d), free(r->best_effort_q), free(r->best_effort_d);
    r->alignment_q = r->alignment_d = r->best_effort_q = r->best_effort_d = nullptr;
}

int aw_align_sliding_window_batch(int n, const char *const *query, const int64_t *qlen, const char *const *reference,
                                  const int64_t *rlen, const int64_t *window, int32_t match, int32_t mis, int32_t o1,
                                  int32_t e1, int32_t o2, int32_t e2, aw_window_result_t *out) {
    if (n < 0 || (n > 0 && (!query || !qlen || !reference || !rlen || !out || !window))) return AW_E_INVAL;
    for (int i = 0; i < n; ++i) {
        if (window[i] <= 0) return AW_E_INVAL;
        if (window[i] > 1073741824) {
            set_error("aw_align_sliding_window_batch: the windows size is too large");
            return AW_E_INVAL;
        }
    }
    std::vector<std::string> Q(n), D(n), AQ(n), AD(n);
    std::vector<int64_t> qs(n, 1), ds(n, 1);
    std::vector<char> whole(n, 0);
    for (int i = 0; i < n; ++i) {
        if (qlen[i] < 0 || rlen[i] < 0 || qlen[i] > INT32_MAX / 2 || rlen[i] > INT32_MAX / 2) return AW_E_INVAL;
        Q[i].assign(query[i] ? query[i] : "", (size_t)qlen[i]);
        D[i].assign(reference[i] ? reference[i] : "", (size_t)rlen[i]);
        whole[i] = ((double)rlen[i] / (double)window[i]) * ((double)qlen[i] / (double)window[i]) <= 1.0;
    }
    // the windows' penalties (:531-535)
    int wm, wo1, we1, wo2, we2;
    if (e2 + match < 0) wm = mis + match, wo1 = o1 + match, we1 = e1 + match, wo2 = o2 + match, we2 = e2 + match;
    else wm = mis + match - 1, wo1 = o1 + match - 1, we1 = e1 + match - 1, wo2 = o2 + match - 1, we2 = -1;
    int rc = AW_OK;
    try {
        // intervals inside the window envelope: minimap2AlignmentWithArena (:490-496)
        std::vector<Job> jobs;
        for (int i = 0; i < n; ++i)
            if (whole[i]) jobs.push_back(Job{i, Q[i], D[i], -1});
        if (!jobs.empty()) {
            std::vector<ksw_extz_t> res;
            rc = run_round(jobs, mis, o1, e1, o2, e2, 0, res);
            for (size_t k = 0; rc == AW_OK && k < jobs.size(); ++k) {
                const int i = jobs[k].id;
                int64_t qp, tp;
                rows(res[k], Q[i], D[i], AQ[i], AD[i], qp, tp);
                qs[i] = qlen[i] + 1, ds[i] = rlen[i] + 1;
            }
            free_ez(res);
        }
        // windows (:497-555): the k-th window of every interval still advancing, in one round
        while (rc == AW_OK) {
            jobs.clear();
            for (int i = 0; i < n; ++i) {
                if (whole[i] || !(ds[i] <= rlen[i] && qs[i] <= qlen[i])) continue;
                // getSubsequence(seq, start, start + W): 1-based, inclusive, clamped at the end
                const int64_t W = window[i];
                const int64_t qe = std::min<int64_t>(qs[i] + W, qlen[i]), de = std::min<int64_t>(ds[i] + W, rlen[i]);
                jobs.push_back(Job{i, Q[i].substr((size_t)qs[i] - 1, (size_t)(qe - qs[i] + 1)),
                                   D[i].substr((size_t)ds[i] - 1, (size_t)(de - ds[i] + 1)), -1});
            }
            if (jobs.empty()) break;
            std::vector<ksw_extz_t> res;
            rc = run_round(jobs, wm, wo1, we1, wo2, we2, AW_EZ_SEMIGLOBAL_END, res);
            for (size_t k = 0; rc == AW_OK && k < jobs.size(); ++k) {
                const Job &J = jobs[k];
                const ksw_extz_t &z = res[k];
                // alignmentMinimap2WithArena's end point (:392-398): the better of the last row and column
                int64_t et, eq;
                if (z.mqe > z.mte) et = z.mqe_t + 1, eq = (int64_t)J.q.size();
                else et = (int64_t)J.d.size(), eq = z.mte_q + 1;
                std::string a, b;
                int64_t qp, tp;
                rows(z, J.q, J.d, a, b, qp, tp);
                if (qp != eq || tp != et) throw std::runtime_error("KSW2 semiglobal traceback did not reconstruct its reported endpoint");
                AQ[J.id] += a, AD[J.id] += b;
                qs[J.id] += eq, ds[J.id] += et;
            }
            free_ez(res);
        }
    } catch (const std::exception &ex) {
        set_error((std::string("aw_align_sliding_window_batch: ") + ex.what()).c_str());
        rc = AW_E_INVAL;
    }
    for (int i = 0; i < n; ++i) {
        aw_window_result_t &o = out[i];
        memset(&o, 0, sizeof(o));
        if (rc != AW_OK) continue;
        // the trailing gaps (:560-575), then the whole alignment re-scored (:585-589)
        const int64_t c1 = rlen[i] - ds[i];
        if (c1 >= 0) AQ[i].append((size_t)(c1 + 1), '-'), AD[i].append(D[i], (size_t)(ds[i] - 1), (size_t)(c1 + 1));
        const int64_t c2 = qlen[i] - qs[i];
        if (c2 >= 0) AQ[i].append(Q[i], (size_t)(qs[i] - 1), (size_t)(c2 + 1)), AD[i].append((size_t)(c2 + 1), '-');
        try {
            o.score = rescore(AQ[i], AD[i], mis, o1, e1, o2, e2);
        } catch (const std::exception &ex) {
            set_error((std::string("aw_align_sliding_window_batch: ") + ex.what()).c_str());
            rc = AW_E_INVAL;
            continue;
        }
        o.alignment_q = dup(AQ[i]), o.alignment_d = dup(AD[i]), o.alignment_len = (int64_t)AQ[i].size();
    }
    return rc;
}

void aw_window_result_free(aw_window_result_t *r) {
    if (!r) return;
    free(r->alignment_q), free(r->alignment_d);
    r->alignment_q = r->alignment_d = nullptr;
}

}  // extern "C"
