// Lattice tables of the D2Q9 and D3Q19 velocity sets in the reference's
// order (SetupD2Q9Latt / SetupD3Q19Latt, Src/model.cpp:99-131) and the
// opposite-direction map (FindReverseXi, Src/model.cpp:82-97).  The
// integer tables are constexpr so that fully unrolled device loops fold
// them into immediates.
#pragma once

#if defined(__CUDACC__)
#define MPLB_HD __host__ __device__ __forceinline__
#else
#define MPLB_HD inline
#endif

namespace mplb {

template <int D>
struct Lattice;

template <>
struct Lattice<2> {
    static constexpr int Q = 9;
    static constexpr int D = 2;
    static MPLB_HD constexpr int cx(int i) {
        return i == 0 ? 0 : i == 1 ? -1 : i == 2 ? -1 : i == 3 ? -1
             : i == 4 ? 0 : i == 5 ? 1 : i == 6 ? 1 : i == 7 ? 1 : 0;
    }
    static MPLB_HD constexpr int cy(int i) {
        return i == 0 ? 0 : i == 1 ? 1 : i == 2 ? 0 : i == 3 ? -1
             : i == 4 ? -1 : i == 5 ? -1 : i == 6 ? 0 : i == 7 ? 1 : 1;
    }
    static MPLB_HD constexpr int cz(int) { return 0; }
    static MPLB_HD constexpr int opp(int i) {
        return i == 0 ? 0 : (i <= 4 ? i + 4 : i - 4);
    }
    // 0: 4/9, 1: 1/9, 2: 1/36 (weight class of direction i)
    static MPLB_HD constexpr int wclass(int i) {
        return i == 0 ? 0 : ((i & 1) ? 2 : 1);
    }
};

template <>
struct Lattice<3> {
    static constexpr int Q = 19;
    static constexpr int D = 3;
    static MPLB_HD constexpr int cx(int i) {
        return (i == 1 || i == 4 || i == 5 || i == 6 || i == 7) ? -1
             : (i == 10 || i == 13 || i == 14 || i == 15 || i == 16) ? 1 : 0;
    }
    static MPLB_HD constexpr int cy(int i) {
        return (i == 2 || i == 4 || i == 8 || i == 9 || i == 14) ? -1
             : (i == 5 || i == 11 || i == 13 || i == 17 || i == 18) ? 1 : 0;
    }
    static MPLB_HD constexpr int cz(int i) {
        return (i == 3 || i == 6 || i == 8 || i == 16 || i == 18) ? -1
             : (i == 7 || i == 9 || i == 12 || i == 15 || i == 17) ? 1 : 0;
    }
    static MPLB_HD constexpr int opp(int i) {
        return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9);
    }
    // 0: 1/3, 1: 1/18, 2: 1/36
    static MPLB_HD constexpr int wclass(int i) {
        return i == 0 ? 0 : ((i <= 3 || (i >= 10 && i <= 12)) ? 1 : 2);
    }
};

template <typename L>
MPLB_HD constexpr int comp(int i, int axis) {
    return axis == 0 ? L::cx(i) : axis == 1 ? L::cy(i) : L::cz(i);
}

}  // namespace mplb
