// ref_checks.cpp -- test infrastructure: the reference's CPU verification of
// its binning (engine/testing.h), restated for the oracle library.
//
// storeGridCellMap (testing.h:25-32) counts every cell id of the unsorted
// keys in an ordered map.  validateGridCellOrdering (testing.h:34-53) walks
// the sorted keys, stops at the first key smaller than its predecessor
// (testing.h:40-43 prints and exits there), counts the sorted keys in a second
// map and reports every cell whose two counts differ (testing.h:48-52).  Both
// run on one host thread with std::map, as the reference's do.
#include <cstdint>
#include <map>

extern "C" {

// Returns 0 when the sorted keys are ordered and every cell's count matches
// the unsorted keys' count; 1 + i when sorted[i] < sorted[i - 1]; -m when m
// cells differ in count.  *cells_out: the number of distinct cells stored.
int64_t orc_ref_grid_cell_checks(const uint32_t* unsorted, const uint32_t* sorted, uint64_t n, uint64_t* cells_out) {
    std::map<uint32_t, uint32_t> grid_map;  // storeGridCellMap
    for (uint64_t i = 0; i < n; ++i) ++grid_map[unsorted[i]];
    if (cells_out) *cells_out = grid_map.size();
    // validateGridCellOrdering
    uint32_t prev = 0;
    std::map<uint32_t, uint32_t> temp_map;
    for (uint64_t i = 0; i < n; ++i) {
        if (prev > sorted[i]) return (int64_t)(i + 1);
        ++temp_map[sorted[i]];
        prev = sorted[i];
    }
    int64_t differ = 0;
    for (auto it = grid_map.begin(); it != grid_map.end(); ++it)
        if (it->second != temp_map[it->first]) ++differ;
    return -differ;
}

}  // extern "C"
