// Shape and weight layout of the learned far-field network (the solver
// MMS_SOLVER_SURROGATE and the mms_farnet_* training entry points).
//
// Leaf boxes of FN_S x FN_S cells x FN_Z layers (cell c = z*64 + y*8 + x);
// FN_NE channels even and FN_NO odd under z -> -z; every translation table is
// block diagonal, one [even NE x NE | odd NO x NO] pair of input-major
// ([j][k]: j input, k output) blocks per operator.  Weight vector (FP32):
//   W    [C][NR]                   encoder            at fn_off_W()
//   V    [NR][C]                   decoder            at fn_off_V()
//   M2L  [depths][49][OSZ]         offset slot (oy + 3) * 7 + (ox + 3),
//                                  o = target - source; the 9 near slots zero
//   then for depth 1 .. depths-1:  M2M [4][OSZ] (child -> this depth's box)
//                                  L2L [4][OSZ] (this depth's box -> child)
// Depth 0 is the leaf level; a grid with L quadtree levels uses depth L - l
// at level l.
//
// Two widths run in the solver (chosen by the length of the weight vector):
//   24 = 16 even + 8 odd: the default, trained by the mms_farnet_* kernels;
//   40 = 24 even + 16 odd: the accurate one, 5-10x closer to the exact sum
//        for a ~30 % longer evaluation (its nested-SVD start, untrained).
// FN_NE / FN_NO are the trainable (default) width.
#pragma once

constexpr int FN_S = 8, FN_Z = 3, FN_C = FN_S * FN_S * FN_Z;
constexpr int FN_NE = 16, FN_NO = 8, FN_NR = FN_NE + FN_NO;
constexpr int FN_OSZ = FN_NE * FN_NE + FN_NO * FN_NO;
constexpr int FN_DEPTHS = 5;
constexpr int FN_NR_MAX = 40;  // widest network the solver runs

// weight layout of a network with NR_ channels, NE_ of them even
template <int NR_, int NE_>
struct FnShape {
    static constexpr int NR = NR_, NE = NE_, NO = NR_ - NE_, OSZ = NE_ * NE_ + (NR_ - NE_) * (NR_ - NE_);
    __host__ __device__ static constexpr long long off_W() { return 0; }
    __host__ __device__ static constexpr long long off_V() { return (long long)FN_C * NR; }
    __host__ __device__ static constexpr long long off_M2L(int d) { return 2LL * FN_C * NR + (long long)d * 49 * OSZ; }
    __host__ __device__ static constexpr long long off_M2M(int d)
    {
        return off_M2L(FN_DEPTHS) + (long long)(d - 1) * 8 * OSZ;
    }
    __host__ __device__ static constexpr long long off_L2L(int d) { return off_M2M(d) + 4LL * OSZ; }
    __host__ __device__ static constexpr long long num_params() { return off_M2M(FN_DEPTHS); }
};
using FnTrain = FnShape<FN_NR, FN_NE>;  // the trainable width
using FnWide = FnShape<40, 24>;         // the accurate width

__host__ __device__ constexpr long long fn_off_W() { return FnTrain::off_W(); }
__host__ __device__ constexpr long long fn_off_V() { return FnTrain::off_V(); }
__host__ __device__ constexpr long long fn_off_M2L(int d) { return FnTrain::off_M2L(d); }
__host__ __device__ constexpr long long fn_off_M2M(int d) { return FnTrain::off_M2M(d); }
__host__ __device__ constexpr long long fn_off_L2L(int d) { return FnTrain::off_L2L(d); }
__host__ __device__ constexpr long long fn_num_params() { return FnTrain::num_params(); }
