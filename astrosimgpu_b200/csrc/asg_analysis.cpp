// Calcium-transient statistics of recorded astrocyte traces, with the
// semantics of the reference's analysis (analysis.cpp:10-220, driven as in
// main.cpp:266-315): threshold events with merging of short gaps, sliding-
// window event rates, pairwise Pearson correlation over cells with at least
// one event, and duration summary.  Host code; the long-run parity
// statistics (active astrocytes, mean pairwise correlation) come from here.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "asg_common.hpp"

namespace asg {

namespace {

struct Events {
    std::vector<double> on, off, dur;
};

// Onsets at the first sample >= threshold, offsets at the last sample above
// it; events running at either edge are kept; gaps shorter than max_gap merge.
Events threshold_events(const double* t, const double* v, std::size_t n, double thr, double gap) {
    Events e;
    if (n < 2) return e;
    for (std::size_t i = 1; i < n; ++i) {
        if (v[i] >= thr && v[i - 1] < thr) e.on.push_back(t[i]);
        if (v[i] < thr && v[i - 1] >= thr) e.off.push_back(t[i - 1]);
    }
    if (v[0] >= thr) e.on.insert(e.on.begin(), t[0]);
    if (v[n - 1] >= thr) e.off.push_back(t[n - 1]);
    if (!e.on.empty() && !e.off.empty()) {
        std::vector<double> on{e.on.front()}, off;
        const std::size_t pairs = std::min(e.on.size(), e.off.size());
        for (std::size_t i = 0; i + 1 < pairs; ++i) {
            if (e.on[i + 1] - e.off[i] >= gap) {
                off.push_back(e.off[i]);
                on.push_back(e.on[i + 1]);
            }
        }
        off.push_back(e.off.back());
        e.on.swap(on);
        e.off.swap(off);
    }
    const std::size_t pairs = std::min(e.on.size(), e.off.size());
    for (std::size_t i = 0; i < pairs; ++i) {
        const double d = e.off[i] - e.on[i];
        if (d >= 0.0) e.dur.push_back(d);
    }
    return e;
}

// Events per ms in windows [start + i*shift, start + i*shift + width].
std::vector<double> window_rates(std::vector<double> ev, double start, double end, double width,
                                 double shift) {
    std::vector<double> h;
    if (shift <= 0.0 || width <= 0.0 || end <= start) return h;
    const auto bins = static_cast<std::int64_t>(std::floor((end - start - width) / shift));
    if (bins <= 0) return h;
    h.assign(static_cast<std::size_t>(bins), 0.0);
    if (ev.empty()) return h;
    std::sort(ev.begin(), ev.end());
    for (std::int64_t i = 0; i < bins; ++i) {
        const double lo = start + static_cast<double>(i) * shift, hi = lo + width;
        const auto a = std::lower_bound(ev.begin(), ev.end(), lo);
        const auto b = std::upper_bound(ev.begin(), ev.end(), hi);
        h[static_cast<std::size_t>(i)] = static_cast<double>(b - a) / width;
    }
    return h;
}

double correlation(const std::vector<double>& a, const std::vector<double>& b) {
    const std::size_t n = std::min(a.size(), b.size());
    if (n < 2) return 0.0;
    double ma = 0.0, mb = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        ma += a[i];
        mb += b[i];
    }
    ma /= static_cast<double>(n);
    mb /= static_cast<double>(n);
    double c = 0.0, va = 0.0, vb = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        const double da = a[i] - ma, db = b[i] - mb;
        c += da * db;
        va += da * da;
        vb += db * db;
    }
    if (va <= 0.0 || vb <= 0.0) return 0.0;
    return c / std::sqrt(va * vb);
}

}  // namespace

}  // namespace asg

extern "C" int asg_calcium_analysis(const double* times, const double* ca, int32_t n_cells,
                                    int32_t n_samples, double threshold, double merge_gap,
                                    double win_start, double win_end, double width, double shift,
                                    double* out5) {
    asg::clear_error();
    if (out5 == nullptr || n_cells < 0 || n_samples < 0 ||
        (n_cells > 0 && n_samples > 0 && (times == nullptr || ca == nullptr)))
        return asg::fail(ASG_ERR_ARG, "asg_calcium_analysis: bad arguments");
    std::vector<std::vector<double>> hists(static_cast<std::size_t>(n_cells));
    std::vector<char> usable(static_cast<std::size_t>(n_cells), 0);
    std::vector<double> durations;
    double active = 0.0;
    for (int32_t c = 0; c < n_cells; ++c) {
        const std::size_t off = static_cast<std::size_t>(c) * n_samples;
        const asg::Events e =
            asg::threshold_events(times + off, ca + off, static_cast<std::size_t>(n_samples),
                                  threshold, merge_gap);
        durations.insert(durations.end(), e.dur.begin(), e.dur.end());
        if (!e.on.empty()) active += 1.0;
        hists[c] = asg::window_rates(e.on, win_start, win_end, width, shift);
        double s = 0.0;
        for (double v : hists[c]) s += v;
        usable[c] = s > 0.0;
    }
    double sum = 0.0, pairs = 0.0;
    for (int32_t i = 0; i + 1 < n_cells; ++i) {
        if (!usable[i]) continue;
        for (int32_t j = i + 1; j < n_cells; ++j) {
            if (!usable[j]) continue;
            sum += asg::correlation(hists[i], hists[j]);
            pairs += 1.0;
        }
    }
    double mean_dur = 0.0;
    if (!durations.empty()) {
        for (double d : durations) mean_dur += d;
        mean_dur /= static_cast<double>(durations.size());
    }
    out5[0] = active;
    out5[1] = static_cast<double>(durations.size());
    out5[2] = mean_dur;
    out5[3] = pairs;
    out5[4] = pairs > 0.0 ? sum / pairs : 0.0;
    return ASG_OK;
}
