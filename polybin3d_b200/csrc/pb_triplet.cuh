// Work-item table shared by the CUDA-core and tensor-core triplet contractions.
#pragma once
#include <array>
#include <cstring>
#include <vector>
#include "pb_common.cuh"

namespace pb {

constexpr int TRIP_TB = 4;  // B maps per item
constexpr int TRIP_TC = 8;  // C maps per item

struct TripletItem {
    int32_t a;
    int32_t b[TRIP_TB];
    int32_t c[TRIP_TC];
    int32_t out[TRIP_TB][TRIP_TC];  // triplet index or -1
};

// Pair rows of the tensor-core form: the distinct (i1, i2) of the triplet list in
// lexicographic order; groups of up to TC_GROUP consecutive pairs share i1.
constexpr int TC_GROUP = 4;
struct TcGroup {
    int32_t a;      // map index of the shared first factor
    int32_t row0;   // first pair row
    int32_t count;  // pairs in the group (<= TC_GROUP)
    int32_t pad;
};

// Device table: [items][pairs (i1,i2)][groups][tmap (row, col) per triplet], 16-byte aligned
struct TableLayout {
    size_t off_items, off_pairs, off_groups, off_tmap, bytes;
};
TableLayout table_layout(const int32_t *counts);  // counts = {n_items, n_pairs, n_groups, n_trip}

int triplet_build_items(int n_a, int n_b, int n_c, const int32_t *idx, int n_trip, std::vector<TripletItem> &items);
int triplet_tc_workspace_size(int64_t n_vox, const int32_t *counts, int n_c, size_t *bytes);
int launch_triplet_tc(const void *A, int n_a, const void *B, int n_b, const void *C, int n_c, int64_t n_vox,
                      const unsigned char *table, const int32_t *counts, double scale, double *out, void *workspace,
                      size_t workspace_bytes, cudaStream_t s);
// the same contraction with A = B = C = one tiled map set (tiled_factor_byte, tiled_c_byte);
// pair factors are among its first n_factor maps
int launch_triplet_tc_tiled(const char *maps, int n_maps, int n_factor, int64_t n_vox, const unsigned char *table,
                            const int32_t *counts, double scale, double *out, void *workspace, size_t workspace_bytes,
                            cudaStream_t s);

}  // namespace pb
