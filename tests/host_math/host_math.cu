// host_math.cu -- the engine's MCG_HD arithmetic (smoothing, barrier bridge,
// streaming payoffs) compiled for the host, so the CPU test suite can compare
// it with the oracle.  Test infrastructure: built by tests/test_device_math_host.py.
#include "../../rust-pricing-library_b200/csrc/mcg_payoff.cuh"

using namespace mcg;

extern "C" {

void hm_smoothing(double h, double input, double* out) {
    double comp;
    const SmoothD ind = smooth_indicator(h, input, comp);
    const SmoothD pos = smooth_positive_part(h, input);
    out[0] = ind.value;
    out[1] = ind.first;
    out[2] = comp;
    out[3] = pos.value;
    out[4] = pos.first;
}

// Continuous barrier over one state sequence, as the path kernels stream it.
int hm_barrier_path(int up, double barrier, double h, const double* states, const double* variances,
                    const double* times, unsigned count, double* survival, double* diag) {
    ProductParams p{};
    p.kind = MCG_PRODUCT_CONTINUOUS_BARRIER;
    p.barrier_direction = up ? MCG_BARRIER_UP : MCG_BARRIER_DOWN;
    p.barrier = barrier;
    ProductAcc s;
    acc_init(s);
    bool failed = false;
    barrier_begin(p, s, h, states[0], failed);
    for (unsigned i = 1; i < count; ++i)
        barrier_interval(p, s, h, states[i - 1], states[i], variances[i - 1], variances[i],
                         times[i] - times[i - 1], failed);
    *survival = barrier_finish(s, h, count - 1, diag);
    return failed ? 1 : 0;
}

void hm_interval_adjoint(int up, double barrier, double h, double lsa, double ls, double rs, double lv,
                         double rv, double dt, double* out) {
    const IntervalAdjoint a = barrier_interval_adjoint(up != 0, barrier, h, lsa, ls, rs, lv, rv, dt);
    out[0] = a.left_state;
    out[1] = a.right_state;
    out[2] = a.left_var;
    out[3] = a.right_var;
}

}  // extern "C"
