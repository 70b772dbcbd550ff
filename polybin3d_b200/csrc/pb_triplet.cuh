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

int triplet_build_items(int n_a, int n_b, int n_c, const int32_t *idx, int n_trip, std::vector<TripletItem> &items);
int triplet_tc_workspace_size(int64_t n_vox, int n_items, int n_trip, size_t *bytes);
int launch_triplet_tc(const void *A, int n_a, const void *B, int n_b, const void *C, int n_c, int64_t n_vox,
                      const TripletItem *items, int n_items, int n_trip, double scale, double *out,
                      void *workspace, size_t workspace_bytes, cudaStream_t s);

}  // namespace pb
