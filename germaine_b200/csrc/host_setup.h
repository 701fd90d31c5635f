/* Host-side per-frequency set-up (see host_setup.c). */
#ifndef GM_HOST_SETUP_H
#define GM_HOST_SETUP_H
#ifdef __cplusplus
extern "C" {
#endif
void gmh_fd_weights(float dh, float w[6]);
void gmh_pml(int nx, int ny, float dh, int npml, int free_surf, float a0_pml, float s,
             float freq, float *out);
void gmh_assembly_scalars(int physics, float freq, float s, float om2[2], float om[2], float om2mu0[2]);
void gmh_source_amp(int physics, float freq, float s, float dh, double amp[2]);
void gmh_wavelet_amp(const float a[2], float dh, double amp[2]);
void gmh_stf_dft(const float *samples, int ns, int ndt, int physics, float freq, float amp[2]);
void gmh_gradient_scalars(int physics, float freq, float s, float om2[2], float om[2]);
double gmh_hess_green_amp(int physics, float dh);
void gmh_stf_unit(const float stf[2], float unit[2]);
void gmh_wiener(const float num[2], const float den[2], float wien[2]);
void gmh_grad_frame(int nx, int ny, int npml, int free_surf, float *coef, unsigned char *passes);
int gmh_gauss_kernel(float dh, float vref, float fc_low, float fsg, float fsg1, int hfs[2], float *w, int wmax);
float gmh_srt_coef(int ix, int iy, float dh, float xc, float yc, float radius);
void gmh_srt_range(float c, float radius, float dh, int n, int *lo, int *hi);
void gmh_taper_grad_shot(int nx, int ny, float dh, float radius, const float *sx, const float *sy, int ntr,
                         const int *rx, const int *ry, int ishot, float *grid);
void gmh_taper_grad_shot1(int nx, int ny, float dh, int filtsize, int nshots, const float *sx, const float *sy,
                          int ntr, const int *rx, const int *ry, float *grid, unsigned char *mark);
float gmh_tikhonov_cost_te(int nx, int ny, int idx, int idy, float dh, float norm1, float norm2, float beta1,
                           float beta2, float lambda1, float lambda2, const float *sigma, const float *epsilon,
                           float l2, float *work);
void gmh_tikhonov_grad_te(int nx, int ny, int idx, int idy, float dh, float norm1, float norm2, float beta1,
                          float beta2, float lambda1, float lambda2, const float *sigma, const float *epsilon,
                          float *grad_sigma, float *grad_epsilon, float *work);
void gmh_srt_receiver_product(int nx, int ny, float dh, float radius, int ntr, const int *rx, const int *ry,
                              double *prod);
#ifdef __cplusplus
}
#endif
#endif
