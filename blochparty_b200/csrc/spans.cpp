// Host-side launch loop of a forward whose recurring pulses are replaced (simulate(..., pulses="reuse") and
// pulses="surrogate"): the windows between occurrences through bp_forward, each occurrence through its map or
// network, all issued from host code in one call. Replaces the per-occurrence dispatch of blochparty's driver
// (engines/gpu/driver.py:617-698 with the reuse branch of bloch_chunk_mma, engines/gpu/cuda/kernels.cu.in:141-165).
#include "../../include/blochparty_b200.h"

extern "C" int bp_forward_spans(const float* spins, const float* sens, int n, int n_coils, const void* segs,
                                const double* seg64, const int32_t* windows, const int32_t* ranges, int n_spans,
                                const BpSpan* spans, float* state, double* raw, int max_ctas, int32_t* status,
                                void* stream) {
    if (!spins || !sens || !segs || !seg64 || !windows || !ranges || !state || !status || n < 1 || n_spans < 0 ||
        (n_spans > 0 && !spans))
        return BP_E_ARG;
    auto step = [&](int r) {
        const int wa = ranges[2 * r], wb = ranges[2 * r + 1];
        if (wb < wa || wa < 0) return BP_E_ARG;
        if (wb == wa) return BP_OK;
        return bp_forward(spins, sens, n, n_coils, segs, seg64, windows, wa, wb, state, raw, nullptr, 1, max_ctas,
                          status, stream);
    };
    for (int i = 0; i < n_spans; ++i) {
        int code = step(i);
        if (code != BP_OK) return code;
        const BpSpan& sp = spans[i];
        switch (sp.kind) {
            case BP_SPAN_MAP:
                code = bp_pulse_apply(sp.map, n, state, sp.phase, stream);
                break;
            case BP_SPAN_NET_MMA:
                code = bp_surrogate_pulse_mma(spins, state, n, sp.params, sp.wtiles, segs, sp.seg0, sp.k_steps, sp.T,
                                              sp.gz, sp.thickness, sp.z0, sp.phase, sp.b0off, sp.dom_df, sp.dom_b1,
                                              sp.dom_z, sp.counts, status, max_ctas, stream);
                break;
            case BP_SPAN_NET_F32:
                code = bp_surrogate_pulse(spins, state, n, sp.params, segs, sp.seg0, sp.k_steps, sp.T, sp.gz,
                                          sp.thickness, sp.z0, sp.phase, sp.b0off, sp.dom_df, sp.dom_b1, sp.dom_z,
                                          sp.counts, stream);
                break;
            default:
                code = BP_E_ARG;
        }
        if (code != BP_OK) return code;
    }
    return step(n_spans);
}
