// entry.h — internal implementations behind the reference-named entry points.
// Shared by the extern "C" definitions (dropin.cpp) and the C++-linkage
// copies (compat_cxx.cpp); it must not include sbb_spmv.h, whose extern "C"
// declarations use the same names.
#pragma once

namespace sbb {
int dropin_baseline(int m, int n, long long nnz, double *alpha, double *val, long long *rp,
                    int *col, double *x, double *beta, double *y, int ngpu);
int dropin_v1(int m, int n, long long nnz, double *alpha, double *val, long long *rp, int *col,
              double *x, double *beta, double *y, int ngpu, int kernel);
int dropin_v2(int m, int n, long long nnz, double *alpha, double *val, long long *rp, int *col,
              double *x, double *beta, double *y, int ngpu, int kernel, long long nb, int q);
int csr5_entry(int m, int n, int nnz, double *alpha, double *val, int *rp, int *col, double *x,
               double *beta, double *y);
int row_from_index(int n, const long long *a, long long idx);
double wall_time();
double min_free_gb(int ngpu);
}  // namespace sbb
