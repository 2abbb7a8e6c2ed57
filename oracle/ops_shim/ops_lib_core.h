/*
 * Sequential stand-in for the OPS structured-mesh library, written for this
 * project so that the reference solver's own sources (Src/*.cpp, Src/*.inc)
 * compile unmodified on a machine without OPS.  TEST INFRASTRUCTURE ONLY:
 * nothing under oracle/ is part of the product path.
 *
 * Only the subset of the OPS API that the reference calls is provided
 * (block/dat/stencil/halo/reduction declarations, ops_par_loop, halo
 * transfer, reductions, timers, printf).  Semantics follow OPS's sequential
 * back end as the reference uses it:
 *   - every ops_dat is allocated with its halo (d_m..size+d_p per axis) and
 *     zero filled (the reference relies on that, Src/type.h:67-68);
 *   - ops_par_loop visits the half-open range with i fastest, then j, then k;
 *   - ops_halo_transfer copies each halo box of the group in declaration
 *     order, all components of every point (Src/field.h:215-395);
 *   - an OPS_INC reduction accumulates sequentially into its handle until
 *     ops_reduction_result returns the value and resets it.
 * Arrays are stored point-major with components contiguous (OPS's default
 * AoS layout), which is invisible through ACC<T>.
 */
#ifndef OPS_LIB_CORE_H
#define OPS_LIB_CORE_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <ostream>
#include <type_traits>

#if !defined(OPS_2D) && !defined(OPS_3D)
#error "define OPS_2D or OPS_3D"
#endif

#define OPS_READ 0
#define OPS_WRITE 1
#define OPS_RW 2
#define OPS_INC 3
#define OPS_MIN 4
#define OPS_MAX 5

#define OPS_ARG_DAT 0
#define OPS_ARG_GBL 1
#define OPS_ARG_IDX 2
#define OPS_ARG_REDUCE 3

#ifndef OPS_FUN_PREFIX
#define OPS_FUN_PREFIX
#endif

struct ops_block_core {
    int dims;
    std::string name;
};
typedef ops_block_core* ops_block;

struct ops_dat_core {
    ops_block block;
    int dim;            // components per point
    int elem_size;      // bytes per component
    int size[3];        // interior points per axis
    int d_m[3];         // (negative) lower halo depth
    int d_p[3];         // upper halo depth
    int alloc[3];       // points allocated per axis
    std::vector<char> data;
    std::string type;
    std::string name;
};
typedef ops_dat_core* ops_dat;

struct ops_stencil_core {
    int dims;
    int points;
    std::string name;
};
typedef ops_stencil_core* ops_stencil;

struct ops_halo_core {
    ops_dat from, to;
    int iter_size[3];
    int from_base[3];
    int to_base[3];
};
typedef ops_halo_core* ops_halo;

struct ops_halo_group_core {
    std::vector<ops_halo> halos;
};
typedef ops_halo_group_core* ops_halo_group;

struct ops_reduction_core {
    double value;
    int size;
    std::string type;
    std::string name;
};
typedef ops_reduction_core* ops_reduction;

struct ops_arg {
    int argtype;
    ops_dat dat;
    char* data;
    int dim;
    int acc;
    ops_reduction red;
};

/* Relative-index accessor handed to each kernel argument that is a dat. */
template <typename T>
class ACC {
   public:
    T* ptr{nullptr};   // component 0 of the current point
    long sx{0}, sy{0}, sz{0};
    int dim{1};
#ifdef OPS_3D
    T& operator()(int d, int i, int j, int k) const {
        return ptr[d + i * sx + j * sy + k * sz];
    }
    T& operator()(int i, int j, int k) const {
        return ptr[i * sx + j * sy + k * sz];
    }
#endif
#ifdef OPS_2D
    T& operator()(int d, int i, int j) const {
        return ptr[d + i * sx + j * sy];
    }
    T& operator()(int i, int j) const { return ptr[i * sx + j * sy]; }
#endif
};

extern FILE* ops_shim_log;
extern int ops_my_global_rank;

void ops_init(const int argc, const char** argv, const int diags_level);
void ops_exit();
ops_block ops_decl_block(int dims, const char* name);
ops_dat ops_decl_dat_char(ops_block block, int dim, int* size, int* base,
                          int* d_m, int* d_p, int elem_size, const char* type,
                          const char* name);
template <typename T>
ops_dat ops_decl_dat(ops_block block, int dim, int* size, int* base, int* d_m,
                     int* d_p, T* /*data*/, const char* type,
                     const char* name) {
    return ops_decl_dat_char(block, dim, size, base, d_m, d_p, sizeof(T),
                             type, name);
}
ops_dat ops_decl_dat_hdf5(ops_block block, int dim, const char* type,
                          const char* name, const char* file);
ops_stencil ops_decl_stencil(int dims, int points, int* sten,
                             const char* name);
ops_halo ops_decl_halo(ops_dat from, ops_dat to, int* iter_size,
                       int* from_base, int* to_base, int* from_dir,
                       int* to_dir);
ops_halo_group ops_decl_halo_group(int nhalos, ops_halo* halos);
void ops_halo_transfer(ops_halo_group group);
ops_reduction ops_decl_reduction_handle(int size, const char* type,
                                        const char* name);
void ops_reduction_result_double(ops_reduction handle, double* result);
template <typename T>
void ops_reduction_result(ops_reduction handle, T* result) {
    ops_reduction_result_double(handle, reinterpret_cast<double*>(result));
}
template <typename T>
void ops_decl_const(const char* /*name*/, int /*dim*/, const char* /*type*/,
                    T* /*data*/) {}
void ops_partition(const char* routine);
void ops_diagnostic_output();
void ops_timing_output(std::ostream& stream);
void ops_timers(double* cpu, double* et);
void ops_printf(const char* format, ...);
void ops_fetch_block_hdf5_file(ops_block block, const char* file);
void ops_fetch_dat_hdf5_file(ops_dat dat, const char* file);

ops_arg ops_arg_dat(ops_dat dat, int dim, ops_stencil stencil,
                    const char* type, int acc);
template <typename T>
ops_arg ops_arg_gbl(T* data, int dim, const char* /*type*/, int acc) {
    ops_arg a;
    a.argtype = OPS_ARG_GBL;
    a.dat = nullptr;
    a.data = reinterpret_cast<char*>(const_cast<typename std::remove_const<T>::type*>(data));
    a.dim = dim;
    a.acc = acc;
    a.red = nullptr;
    return a;
}
ops_arg ops_arg_idx();
ops_arg ops_arg_reduce(ops_reduction handle, int dim, const char* type,
                       int acc);

/* Raw access used by project-side glue and harnesses (same role as OPS's
 * ops_dat_get_raw_pointer): pointer to component 0 of point (0,0[,0]) plus
 * the element strides of the three axes. */
char* ops_shim_point_ptr(ops_dat dat, int i, int j, int k);
/* OPS's copies of a dat's interior points (no halo) to / from a user
 * buffer, point-major with all components of a point together. */
void ops_dat_fetch_data(ops_dat dat, int part, char* data);
void ops_dat_set_data(ops_dat dat, int part, char* data);
long ops_shim_stride(ops_dat dat, int axis);

#endif  // OPS_LIB_CORE_H
