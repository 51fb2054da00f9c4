// unet_guard.h -- outcome monitor of the learned warm start (host code).
//
// Policy only: which solve may start from the network's prediction, and what
// the iteration counts of finished solves say about the network.  Kept free
// of CUDA so that its logic is tested on the CPU.
#pragma once
#include <algorithm>

namespace hc {

// Outcome monitor of the learned warm start.  The acceptance test of a
// prediction (max|delta| decreased) cannot see smooth error, so an accepted
// prediction may still cost iterations.  The monitor compares the SOR
// iterations of consecutive solves of which one started from a prediction and
// the other from the previous potential ("plain": a rejected prediction, a
// probe, or the network switched off).  Plain probe solves are scheduled
// after `period` predicted solves; the period grows with a clear win (the
// prediction needed under a quarter of the plain iterations: 64, doubling to
// 1024) and shrinks to 2 after a loss.  After K consecutive losses the network
// is switched off; it is retried after 16 solves, doubling to 256 after each
// failed retry, and a win switches it back on.  The first solve of a context
// (a cold start) is not compared.
struct UnetGuard {
    int K = 0;                 // consecutive losses that switch the network off (0: monitor off)
    int off = 0;
    int started = 0;           // a solve has run (the cold start is not compared)
    int prev_kind = 0;         // previous solve: 0 none, 1 plain, 2 predicted
    int prev_iters = 0;
    int until_probe = 1;
    int period = 4;
    int retry_gap = 16;
    int until_retry = 0;
    int losses = 0;
    int probe_now = 0;         // this solve is a probe
    int retry_now = 0;         // this solve retries the switched-off network
    long long probes = 0, wins = 0, loss_total = 0, switch_offs = 0;
};

// Whether the solve about to run may start from a prediction.
inline bool unet_guard_allows(UnetGuard &g)
{
    g.probe_now = 0;
    g.retry_now = 0;
    if (g.K <= 0 || !g.started) return true;
    if (g.off) {
        if (--g.until_retry > 0) return false;
        g.retry_now = 1;
        return true;
    }
    if (g.until_probe <= 0) {
        g.probe_now = 1;
        g.probes++;
        return false;
    }
    return true;
}

// Outcome of a finished solve: predicted (a prediction accepted in its first
// cycle) or plain, and its SOR iterations.
inline void unet_guard_record(UnetGuard &g, bool predicted, int iters)
{
    if (g.K <= 0) return;
    const int kind = predicted ? 2 : 1;
    if (!g.started) {   // the cold start
        g.started = 1;
        g.prev_kind = 0;
        return;
    }
    bool won = false;
    if (g.prev_kind != 0 && g.prev_kind != kind) {
        const int n_pred = predicted ? iters : g.prev_iters;
        const int n_plain = predicted ? g.prev_iters : iters;
        if (n_pred < n_plain) {
            const double r = (double)n_pred / std::max(1, n_plain);
            won = true;
            g.wins++;
            g.losses = 0;
            if (g.off) {   // a retry won: back on
                g.off = 0;
                g.retry_gap = 16;
                g.period = 4;
            }
            g.period = r < 0.25 ? std::min(std::max(2 * g.period, 64), 1024) : (r < 0.5 ? 16 : 4);
            g.until_probe = g.period;
        } else {
            g.loss_total++;
            g.losses++;
            g.period = 2;
            g.until_probe = std::min(g.until_probe, g.period);
            if (!g.off && g.losses >= g.K) {
                g.off = 1;
                g.switch_offs++;
                g.retry_gap = 16;
                g.until_retry = g.retry_gap;
            }
        }
    }
    if (g.retry_now && !won) {   // a retry that lost or was rejected
        g.retry_gap = std::min(2 * g.retry_gap, 256);
        g.until_retry = g.retry_gap;
    }
    if (g.probe_now) g.until_probe = std::max(g.until_probe, 1);
    else if (!g.off && predicted) g.until_probe--;
    g.prev_kind = kind;
    g.prev_iters = iters;
}

}  // namespace hc
