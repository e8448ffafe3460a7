/* Stand-in for the absent FFTW3 header (oracle build only).  FFTs are not on
   the ray-shooting path; every routine is a no-op. */
#pragma once
typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;
#define FFTW_ESTIMATE 64
#define FFTW_MEASURE 0
inline fftw_plan fftw_plan_dft_c2r_2d(...) { return nullptr; }
inline fftw_plan fftw_plan_dft_r2c_2d(...) { return nullptr; }
inline void fftw_execute(...) {}
inline void fftw_execute_dft_c2r(...) {}
inline void fftw_execute_dft_r2c(...) {}
inline void fftw_destroy_plan(...) {}
