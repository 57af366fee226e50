// Host-side sizes of the device buffers a simulation needs (no GPU needed): see bp_forward_workspace_bytes and
// bp_adjoint_workspace_bytes in include/blochparty_b200.h. The Python host side allocates exactly these.
#include <cstdint>

#include "../../include/blochparty_b200.h"

extern "C" int bp_forward_workspace_bytes(int n, int64_t n_adc, int n_coils, BpForwardWorkspace* out) {
    if (!out || n < 1 || n_adc < 0 || n_coils < 1 || n_coils > BP_MAX_COILS) return BP_E_ARG;
    const int64_t nn = n, rows = n_adc > 0 ? n_adc : 1;
    out->state = 6 * nn * 4;
    out->raw = rows * 2 * n_coils * 8;
    out->psi = n_adc * 8;
    out->signal = (int64_t)n_coils * rows * 8;
    out->status = 4;
    out->total = out->state + out->raw + out->psi + out->signal + out->status;
    return BP_OK;
}

extern "C" int bp_adjoint_workspace_bytes(int n, int64_t n_segments, int64_t n_adc, int n_coils, int checkpoint_every,
                                          int max_interval_windows, int grid, int outer_every,
                                          BpAdjointWorkspace* out) {
    if (!out || n < 1 || n_segments < 0 || n_adc < 0 || n_coils < 1 || n_coils > BP_MAX_COILS ||
        checkpoint_every < BP_ADJ_WIN || checkpoint_every % BP_ADJ_WIN != 0 || max_interval_windows < 0 || grid < 1 ||
        outer_every < 0)
        return BP_E_ARG;
    const int64_t nn = n, every = checkpoint_every;
    const int64_t intervals = n_segments > 0 ? (n_segments + every - 1) / every : 0;
    const int64_t longest = n_segments < every ? n_segments : every;  // segments of the longest interval
    // with an outer level: the state at every block start, and one block's interval starts
    const int64_t states = outer_every > 1 ? (intervals + outer_every - 1) / outer_every +
                                                 (intervals < outer_every ? intervals : (int64_t)outer_every)
                                           : intervals;
    out->checkpoints = states * 6 * nn * 4;
    out->wstates = ((int64_t)max_interval_windows + 1) * 6 * nn * 4;
    out->replay_state = 6 * nn * 4;
    out->gseg = (int64_t)grid * longest * 8 * 4;
    out->seg = n_segments * 8 * 8;
    out->lam = 3 * nn * 4;
    out->gs = 8 * nn * 4;
    out->gc = 2 * (int64_t)n_coils * nn * 4;
    out->h = n_adc * 2 * n_coils * 4;
    out->total = out->checkpoints + out->wstates + out->replay_state + out->gseg + out->seg + out->lam + out->gs +
                 out->gc + out->h;
    return BP_OK;
}
