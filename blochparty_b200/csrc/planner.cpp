// Host-side window planner of the C ABI (no GPU needed): see bp_plan_windows in include/blochparty_b200.h.
#include <cstdint>

#include "../../include/blochparty_b200.h"

extern "C" int bp_plan_windows(const int32_t* flags, int64_t n_segments, int seg_max, int samp_max,
                               const uint8_t* breaks, int32_t* windows, int64_t max_windows, int64_t* n_windows) {
    if (!flags || !windows || !n_windows || n_segments < 0 || seg_max < 1 || seg_max > BP_SEG_MAX || samp_max < 1)
        return BP_E_ARG;
    int64_t nw = 0, row = 0, s = 0;
    while (s < n_segments) {
        const int64_t start = s, row0 = row;
        int64_t samples = 0;
        bool limited = false;  // cut by seg_max or samp_max (not by a break or the sequence's end)
        while (s < n_segments) {
            if (s > start && breaks && breaks[s]) break;
            const bool adc = (flags[s] & 2) != 0;
            if (s - start == seg_max || (adc && samples == samp_max)) {
                limited = true;
                break;
            }
            samples += adc ? 1 : 0;
            ++s;
        }
        // a limit's cut moves back to a multiple of BP_ADJ_WIN segments when the window keeps one: the cuts then
        // fall on the same segments whatever the breaks before them
        const int64_t aligned = (s / BP_ADJ_WIN) * BP_ADJ_WIN;
        if (limited && aligned > start) {
            for (int64_t t = aligned; t < s; ++t) samples -= (flags[t] & 2) ? 1 : 0;
            s = aligned;
        }
        row += samples;
        if (nw >= max_windows) return BP_E_SIZE;
        windows[4 * nw] = static_cast<int32_t>(start);
        windows[4 * nw + 1] = static_cast<int32_t>(s);
        windows[4 * nw + 2] = static_cast<int32_t>(row0);
        windows[4 * nw + 3] = static_cast<int32_t>(samples);
        ++nw;
    }
    *n_windows = nw;
    return BP_OK;
}
