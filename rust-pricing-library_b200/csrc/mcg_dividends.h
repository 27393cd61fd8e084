// mcg_dividends.h -- the escrowed affine model of discrete dividends, host side.
//
// AffineDividendTransform with carry curves (crates/pricing/src/market/dividend.rs:283-518,
// compile_event :622-642, validation :644-690): each event (ex-time t_k, fixed
// cash c_k, proportional fraction beta_k) removes alpha_k = c_k / S0 of the
// spot scale and a fraction beta_k of the residual.  The funded cash reserve
// R = sum_k c_k / prod_{j<=k}(1 - beta_j) * Dr(t_k) / Dq(t_k) must leave a
// positive residual S0 - R.  The simulated state f is the canonical
// martingale with forward S0 Dq/Dr; an observed spot is A S0 + B f with the
// coordinate (A, B, spot_scale) of the observation time: the initial
// (R / S0, (S0 - R) / S0, 1) carried between events by the growth Dq/Dr of
// the remaining reserve and mapped through every event up to the time, A = 0
// once no cash remains.  The coordinates are plan data: computed once on the
// host and uploaded for the kernels.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace mcg {

struct HostCoord {
    double a = 0.0, b = 1.0, spot_scale = 1.0;
};

template <class Curve>
struct HostDividends {
    struct Event {
        double t, cash, alpha, beta;
    };
    std::vector<Event> ev;
    double spot = 0.0, reserve = 0.0;
    const Curve* rc = nullptr;
    const Curve* qc = nullptr;

    // Validates and compiles the schedule at spot s0; `why` names a failure.
    bool compile(const mcg_dividends& d, double s0, const Curve& r, const Curve& q, std::string& why) {
        ev.clear();
        spot = s0;
        rc = &r;
        qc = &q;
        if (d.count && (!d.ex_times || !d.fixed_cash || !d.proportional)) {
            why = "discrete_dividends: null arrays";
            return false;
        }
        for (uint32_t i = 0; i < d.count; ++i) {
            const double t = d.ex_times[i], cash = d.fixed_cash[i], beta = d.proportional[i];
            if (!std::isfinite(t) || t < 0.0 || (i && !(t > d.ex_times[i - 1]))) {
                why = "discrete_dividends: ex-time " + std::to_string(i) + " must be finite, >= 0 and increasing";
                return false;
            }
            if (!(std::isfinite(cash) && cash >= 0.0)) {
                why = "discrete_dividends: cash " + std::to_string(i) + " must be finite and >= 0";
                return false;
            }
            if (!(std::isfinite(beta) && beta >= 0.0 && beta < 1.0)) {
                why = "discrete_dividends: proportional fraction " + std::to_string(i) + " outside [0, 1)";
                return false;
            }
            const double alpha = cash / s0;
            if (!std::isfinite(alpha)) {
                why = "discrete_dividends: non-finite alpha";
                return false;
            }
            ev.push_back({t, cash, alpha, beta});
        }
        double proportional = 1.0, res = 0.0;
        for (const auto& e : ev) {
            proportional *= 1.0 - e.beta;
            const double discount = std::exp(rc->log_discount(e.t)) / std::exp(qc->log_discount(e.t));
            res += e.cash / proportional * discount;
        }
        const double residual = s0 - res;
        if (!std::isfinite(res) || !std::isfinite(residual) || residual <= 0.0) {
            why = "discrete_dividends: the cash reserve leaves no positive escrowed spot";
            return false;
        }
        reserve = res;
        return true;
    }

    HostCoord initial() const { return {reserve / spot, (spot - reserve) / spot, 1.0}; }

    HostCoord carry(HostCoord c, double start, double end) const {
        if (c.a == 0.0 || start == end) return c;
        const double g = qc->log_discount(end) - rc->log_discount(end) - qc->log_discount(start) +
                         rc->log_discount(start);
        c.a *= std::exp(g);
        return c;
    }

    static HostCoord after(HostCoord c, const Event& e) {
        return {(1.0 - e.beta) * c.a - e.alpha, (1.0 - e.beta) * c.b, (1.0 - e.beta) * c.spot_scale};
    }

    // coordinate_after_time
    HostCoord after_time(double time) const {
        if (ev.empty()) return HostCoord{};
        HostCoord c = initial();
        double prev = 0.0;
        for (const auto& e : ev) {
            if (!(e.t <= time)) break;
            c = carry(c, prev, e.t);
            c = after(c, e);
            prev = e.t;
        }
        c = carry(c, prev, time);
        bool settled = true;
        for (const auto& e : ev) settled = settled && (e.t <= time || e.cash == 0.0);
        if (settled) c.a = 0.0;
        return c;
    }

    // event_timeline's coordinate just before event i
    HostCoord before_event(size_t i) const {
        if (ev.empty()) return HostCoord{};
        HostCoord c = initial();
        double prev = 0.0;
        size_t last_cash = ev.size();
        for (size_t k = ev.size(); k-- > 0;)
            if (ev[k].cash != 0.0) {
                last_cash = k;
                break;
            }
        for (size_t k = 0; k < ev.size(); ++k) {
            const HostCoord before = carry(c, prev, ev[k].t);
            if (k == i) return before;
            HostCoord aft = after(before, ev[k]);
            if (last_cash == ev.size() || k >= last_cash) aft.a = 0.0;
            c = aft;
            prev = ev[k].t;
        }
        return c;
    }

    // index of the event at exactly `time` (bit pattern), or -1
    long event_at(double time) const {
        for (size_t k = 0; k < ev.size(); ++k) {
            uint64_t x, y;
            std::memcpy(&x, &ev[k].t, 8);
            std::memcpy(&y, &time, 8);
            if (x == y) return static_cast<long>(k);
        }
        return -1;
    }
};

}  // namespace mcg
