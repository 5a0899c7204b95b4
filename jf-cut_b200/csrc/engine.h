// engine.h — host-side engine shared by the plain solver, the batch and the
// server (C++ only; not part of the C ABI).
#pragma once

#include <string>
#include <vector>

#include "jfc_internal.h"

struct jfc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;     // the stream every launch of this context uses
  cudaStream_t own_stream = nullptr; // the context's own stream
  jfc_params params{};
  void* h_pin = nullptr;         // pinned host scratch for counter read-back
  size_t h_pin_bytes = 0;
};

// Colour model + inputs kept on the device for warm seed edits.
struct DevModel {
  bool valid = false;
  BuildModelDev m{};
  void* d_img = nullptr;
  uint8_t* d_seeds = nullptr;
  int* d_lut_s = nullptr;        // t-link tables [JFC_TQ + 1]
  int* d_lut_t = nullptr;
  size_t img_bytes = 0;
};

struct jfc_graph {
  jfc_ctx* ctx = nullptr;
  int device = 0;
  int dims = 2, W = 0, H = 0, D = 1, conn = 4;
  GridDev g{};                   // tile fields unset; pointers into d_state
  void* d_state = nullptr;
  size_t state_bytes = 0;
  long long sink_total = 0;      // sum of sink t-link capacities (int64)
  int state = 0;                 // 0 empty, 1 graph loaded, 2 solved
  long long flow = 0;
  long long source_nodes = 0;
  TileSet ts;                    // tile set of this graph alone
  int ts_shape = -1;             // tile shape the tile set was built for
  DevModel model;
  uint8_t* d_dense = nullptr;    // dense scratch for pack / unpack (lazily)
  size_t dense_bytes = 0;
  jfc_stats last{};
};

// Per-grid result of an engine run.
struct GridResult {
  long long neg_sum = 0;
  long long labels = 0;
  int status = JFC_OK;
};

// Solve every grid of `ts` to the exact max-flow (engine.cpp).
int engine_solve(jfc_ctx* ctx, TileSet& ts, const jfc_params& p, std::vector<GridResult>& res,
                 jfc_stats& st);
// Build / free a tile set over grids (all of one dimensionality).
int tileset_build(TileSet& ts, int dims, int tile_rows, const std::vector<GridDev>& grids);
void tileset_free(TileSet& ts);
int shape_code(int dims, int tile_rows);

int set_error(int code, const std::string& msg);
int cuda_status(cudaError_t e, const char* where);
#define JFC_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return cuda_status(_e, #call); \
  } while (0)

void fill_defaults(jfc_params& p);
double elapsed_ms(cudaEvent_t a, cudaEvent_t b);
