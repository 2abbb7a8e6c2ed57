/*
 * ops_par_loop for the sequential OPS stand-in (test infrastructure only).
 *
 * A kernel  void K(P0, P1, ...)  is called once per point of the half-open
 * range, i fastest.  Each parameter is adapted from its ops_arg:
 *   ACC<T>& / const ACC<T>&  <- ops_arg_dat   (positioned at the point)
 *   T* / const T*            <- ops_arg_gbl   (the global's storage)
 *                            <- ops_arg_idx   (int[3] with the point index)
 *                            <- ops_arg_reduce(the handle's accumulator)
 * With OPS_SHIM_OMP defined, loops that carry no reduction run their outer
 * axes under OpenMP; every reference kernel writes only its own point, so the
 * result is identical to the sequential loop.
 */
#ifndef OPS_SEQ_V2_H
#define OPS_SEQ_V2_H
#include <tuple>
#include <utility>
#include "ops_lib_core.h"

namespace ops_shim_detail {

template <typename P>
struct Adapter;

template <typename T>
struct Adapter<ACC<T>&> {
    ACC<T> acc;
    ops_dat dat{nullptr};
    void init(const ops_arg& a) {
        dat = a.dat;
        acc.dim = dat->dim;
        acc.sx = ops_shim_stride(dat, 0);
        acc.sy = ops_shim_stride(dat, 1);
        acc.sz = ops_shim_stride(dat, 2);
    }
    void at(int i, int j, int k) {
        acc.ptr = reinterpret_cast<T*>(ops_shim_point_ptr(dat, i, j, k));
    }
    ACC<T>& get() { return acc; }
};

template <typename T>
struct Adapter<const ACC<T>&> : Adapter<ACC<T>&> {};

template <typename T>
struct Adapter<T*> {
    T* p{nullptr};
    int idx[3]{0, 0, 0};
    bool isIdx{false};
    void init(const ops_arg& a) {
        isIdx = (a.argtype == OPS_ARG_IDX);
        if (a.argtype == OPS_ARG_REDUCE) {
            p = reinterpret_cast<T*>(&a.red->value);
        } else {
            p = reinterpret_cast<T*>(a.data);
        }
    }
    void at(int i, int j, int k) {
        idx[0] = i;
        idx[1] = j;
        idx[2] = k;
    }
    T* get() { return isIdx ? reinterpret_cast<T*>(idx) : p; }
};

template <typename Tuple, std::size_t... I>
inline void InitAll(Tuple& t, const ops_arg* a, std::index_sequence<I...>) {
    (void)std::initializer_list<int>{(std::get<I>(t).init(a[I]), 0)...};
}
template <typename Tuple, std::size_t... I>
inline void AtAll(Tuple& t, int i, int j, int k, std::index_sequence<I...>) {
    (void)std::initializer_list<int>{(std::get<I>(t).at(i, j, k), 0)...};
}
template <typename K, typename Tuple, std::size_t... I>
inline void CallK(K kernel, Tuple& t, std::index_sequence<I...>) {
    kernel(std::get<I>(t).get()...);
}

}  // namespace ops_shim_detail

template <typename... P, typename... A>
void ops_par_loop(void (*kernel)(P...), const char* /*name*/,
                  ops_block /*block*/, int dim, int* range, A... args) {
    static_assert(sizeof...(P) == sizeof...(A),
                  "kernel arity differs from the number of ops_args");
    using namespace ops_shim_detail;
    using Tup = std::tuple<Adapter<P>...>;
    const ops_arg argv[] = {args...};
    Tup tmpl;
    InitAll(tmpl, argv, std::index_sequence_for<P...>{});
    const int imin = range[0], imax = range[1];
    const int jmin = range[2], jmax = range[3];
    const int kmin = dim > 2 ? range[4] : 0;
    const int kmax = dim > 2 ? range[5] : 1;
    bool hasReduction = false;
    for (const ops_arg& a : argv) {
        hasReduction = hasReduction || (a.argtype == OPS_ARG_REDUCE);
    }
#ifdef OPS_SHIM_OMP
    if (!hasReduction) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = kmin; k < kmax; k++) {
            for (int j = jmin; j < jmax; j++) {
                Tup t = tmpl;
                for (int i = imin; i < imax; i++) {
                    AtAll(t, i, j, k, std::index_sequence_for<P...>{});
                    CallK(kernel, t, std::index_sequence_for<P...>{});
                }
            }
        }
        return;
    }
#endif
    (void)hasReduction;
    for (int k = kmin; k < kmax; k++) {
        for (int j = jmin; j < jmax; j++) {
            for (int i = imin; i < imax; i++) {
                AtAll(tmpl, i, j, k, std::index_sequence_for<P...>{});
                CallK(kernel, tmpl, std::index_sequence_for<P...>{});
            }
        }
    }
}

#endif  // OPS_SEQ_V2_H
