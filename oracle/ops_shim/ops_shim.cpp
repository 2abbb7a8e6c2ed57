/*
 * Non-template part of the sequential OPS stand-in (test infrastructure
 * only; see ops_lib_core.h for the semantics it reproduces).
 */
#include "ops_lib_core.h"

#include <chrono>
#include <cstdarg>
#include <ctime>

FILE* ops_shim_log = stdout;
int ops_my_global_rank = 0;

void ops_init(const int /*argc*/, const char** /*argv*/,
              const int /*diags_level*/) {
    const char* quiet = std::getenv("OPS_SHIM_QUIET");
    if (quiet != nullptr && quiet[0] == '1') {
        ops_shim_log = nullptr;
    }
}

void ops_exit() {}

ops_block ops_decl_block(int dims, const char* name) {
    ops_block b = new ops_block_core;
    b->dims = dims;
    b->name = name;
    return b;
}

ops_dat ops_decl_dat_char(ops_block block, int dim, int* size, int* /*base*/,
                          int* d_m, int* d_p, int elem_size, const char* type,
                          const char* name) {
    ops_dat d = new ops_dat_core;
    d->block = block;
    d->dim = dim;
    d->elem_size = elem_size;
    for (int a = 0; a < 3; a++) {
        const bool used = a < block->dims;
        d->size[a] = used ? size[a] : 1;
        d->d_m[a] = used ? d_m[a] : 0;
        d->d_p[a] = used ? d_p[a] : 0;
        d->alloc[a] = d->size[a] + d->d_p[a] - d->d_m[a];
    }
    const size_t points =
        (size_t)d->alloc[0] * (size_t)d->alloc[1] * (size_t)d->alloc[2];
    d->data.assign(points * (size_t)dim * (size_t)elem_size, 0);
    d->type = type;
    d->name = name;
    return d;
}

ops_dat ops_decl_dat_hdf5(ops_block /*block*/, int /*dim*/,
                          const char* /*type*/, const char* name,
                          const char* file) {
    std::fprintf(stderr,
                 "ops shim: restart from HDF5 (%s in %s) is not available\n",
                 name, file);
    std::abort();
}

ops_stencil ops_decl_stencil(int dims, int points, int* /*sten*/,
                             const char* name) {
    ops_stencil s = new ops_stencil_core;
    s->dims = dims;
    s->points = points;
    s->name = name;
    return s;
}

ops_halo ops_decl_halo(ops_dat from, ops_dat to, int* iter_size,
                       int* from_base, int* to_base, int* /*from_dir*/,
                       int* /*to_dir*/) {
    ops_halo h = new ops_halo_core;
    h->from = from;
    h->to = to;
    const int dims = from->block->dims;
    for (int a = 0; a < 3; a++) {
        h->iter_size[a] = a < dims ? iter_size[a] : 1;
        h->from_base[a] = a < dims ? from_base[a] : 0;
        h->to_base[a] = a < dims ? to_base[a] : 0;
    }
    return h;
}

ops_halo_group ops_decl_halo_group(int nhalos, ops_halo* halos) {
    ops_halo_group g = new ops_halo_group_core;
    g->halos.assign(halos, halos + nhalos);
    return g;
}

char* ops_shim_point_ptr(ops_dat d, int i, int j, int k) {
    const size_t ii = (size_t)(i - d->d_m[0]);
    const size_t jj = (size_t)(j - d->d_m[1]);
    const size_t kk = (size_t)(k - d->d_m[2]);
    const size_t point =
        (kk * (size_t)d->alloc[1] + jj) * (size_t)d->alloc[0] + ii;
    return d->data.data() + point * (size_t)d->dim * (size_t)d->elem_size;
}

long ops_shim_stride(ops_dat d, int axis) {
    long s = d->dim;
    for (int a = 0; a < axis; a++) {
        s *= d->alloc[a];
    }
    return s;
}

void ops_halo_transfer(ops_halo_group group) {
    for (ops_halo h : group->halos) {
        const size_t bytes = (size_t)h->from->dim * (size_t)h->from->elem_size;
        for (int k = 0; k < h->iter_size[2]; k++) {
            for (int j = 0; j < h->iter_size[1]; j++) {
                for (int i = 0; i < h->iter_size[0]; i++) {
                    const char* src = ops_shim_point_ptr(
                        h->from, h->from_base[0] + i, h->from_base[1] + j,
                        h->from_base[2] + k);
                    char* dst = ops_shim_point_ptr(h->to, h->to_base[0] + i,
                                                   h->to_base[1] + j,
                                                   h->to_base[2] + k);
                    std::memcpy(dst, src, bytes);
                }
            }
        }
    }
}

ops_reduction ops_decl_reduction_handle(int size, const char* type,
                                        const char* name) {
    ops_reduction r = new ops_reduction_core;
    r->value = 0;
    r->size = size;
    r->type = type;
    r->name = name;
    return r;
}

void ops_reduction_result_double(ops_reduction handle, double* result) {
    *result = handle->value;
    handle->value = 0;
}

void ops_partition(const char* /*routine*/) {}
void ops_diagnostic_output() {}
void ops_timing_output(std::ostream& /*stream*/) {}

void ops_timers(double* cpu, double* et) {
    const double now = std::chrono::duration<double>(
                           std::chrono::steady_clock::now().time_since_epoch())
                           .count();
    *cpu = (double)std::clock() / CLOCKS_PER_SEC;
    *et = now;
}

void ops_printf(const char* format, ...) {
    if (ops_shim_log == nullptr) {
        return;
    }
    va_list ap;
    va_start(ap, format);
    std::vfprintf(ops_shim_log, format, ap);
    va_end(ap);
}

void ops_fetch_block_hdf5_file(ops_block /*block*/, const char* /*file*/) {}
void ops_fetch_dat_hdf5_file(ops_dat /*dat*/, const char* /*file*/) {}

ops_arg ops_arg_dat(ops_dat dat, int dim, ops_stencil /*stencil*/,
                    const char* /*type*/, int acc) {
    ops_arg a;
    a.argtype = OPS_ARG_DAT;
    a.dat = dat;
    a.data = nullptr;
    a.dim = dim;
    a.acc = acc;
    a.red = nullptr;
    return a;
}

ops_arg ops_arg_idx() {
    ops_arg a;
    a.argtype = OPS_ARG_IDX;
    a.dat = nullptr;
    a.data = nullptr;
    a.dim = 0;
    a.acc = OPS_READ;
    a.red = nullptr;
    return a;
}

ops_arg ops_arg_reduce(ops_reduction handle, int dim, const char* /*type*/,
                       int acc) {
    ops_arg a;
    a.argtype = OPS_ARG_REDUCE;
    a.dat = nullptr;
    a.data = nullptr;
    a.dim = dim;
    a.acc = acc;
    a.red = handle;
    return a;
}

void ops_dat_fetch_data(ops_dat d, int /*part*/, char* data) {
    const size_t bytes = (size_t)d->dim * (size_t)d->elem_size;
    for (int k = 0; k < d->size[2]; k++)
        for (int j = 0; j < d->size[1]; j++)
            for (int i = 0; i < d->size[0]; i++) {
                std::memcpy(data, ops_shim_point_ptr(d, i, j, k), bytes);
                data += bytes;
            }
}

void ops_dat_set_data(ops_dat d, int /*part*/, char* data) {
    const size_t bytes = (size_t)d->dim * (size_t)d->elem_size;
    for (int k = 0; k < d->size[2]; k++)
        for (int j = 0; j < d->size[1]; j++)
            for (int i = 0; i < d->size[0]; i++) {
                std::memcpy(ops_shim_point_ptr(d, i, j, k), data, bytes);
                data += bytes;
            }
}
