/*
 * Subset orders of the reference's OS-EM/OS-ART loops — TEST INFRASTRUCTURE
 * ONLY (part of the oracle).  The order comes from libstdc++'s std::shuffle
 * driven by a default-seeded std::mt19937_64, so it is computed here with the
 * same library rather than restated.
 *   IR::reconstruct  (reconstruct.cu:62-81): one engine for the whole run; the
 *                     persistent order is shuffled once per (axis, epoch).
 *   XTT::reconstruct (reconstruct.cu:843-859): a fresh engine every epoch
 *                     shuffles the persistent order.
 */
#include <algorithm>
#include <random>
#include <vector>

extern "C" void or_subset_orders(int batch, int rows, int fresh_engine_each_row, int *out) {
    std::vector<int> order(batch);
    for (int i = 0; i < batch; i++) order[i] = i;
    std::mt19937_64 run_engine;
    for (int r = 0; r < rows; r++) {
        if (fresh_engine_each_row) {
            std::mt19937_64 eng;
            std::shuffle(order.begin(), order.end(), eng);
        } else {
            std::shuffle(order.begin(), order.end(), run_engine);
        }
        std::copy(order.begin(), order.end(), out + (long)r * batch);
    }
}
