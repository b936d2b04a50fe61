/* psm_host.h -- C ABI of libpsm_host.so, the host surface of the B200 migration.
 *
 * The reference (sergeevsn/poststackmig3d) is one executable whose host side is C++ classes:
 * ConfigParser (include/config_parser.h:22-33), SegyFile / SegyOutputFile
 * (include/segy_utils.h:45-166), the VelocityProvider family (include/velocity_reader.h:11-122)
 * and the driver in src/main.cpp:66-442.  This library restates them in C++ and exposes them
 * through the functions below; the compute goes through libpsm_cuda.so (psm.h).  Every call
 * returns PSM_OK (0) or a negative psm_status and fills err (may be NULL) with the message the
 * reference would print after "Error: ".
 */
#ifndef PSM_HOST_H
#define PSM_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Config (include/config_parser.h:7-20; src/config_parser.cpp:74-212).  Strings are
 * NUL-terminated and truncated to the buffer size.  Keys beyond the reference's:
 *   precision   f32 | bf16 | f16   (default f32)  storage of the traces in HBM
 *   compensated bool              (default false) compensated summation
 *   device      int               (default 0)     CUDA device
 *   compat_omp_pad bool           (default false) trailing padded crosslines as the
 *                                 reference's OpenMP build computes them (psm_geom) */
typedef struct {
    char input_data[1024];
    char output_data[1024];
    double inline_step;
    double crossline_step;
    int32_t inline_padding;
    int32_t crossline_padding;
    char velocity[1024];
    double angle_aperture;
    int32_t amp_correction;
    int32_t n_threads;
    int32_t precision;
    int32_t compensated;
    int32_t device;
    int32_t compat_omp_pad;
} psm_config;

/* ConfigParser::parseConfigFile followed by validateConfig. */
int psm_config_load(const char *path, psm_config *out, char *err, size_t err_len);

/* SEG-Y (src/segy_utils.cpp:39-214). */
typedef struct {
    int64_t num_traces;  /* from the file size */
    int32_t num_samples; /* binary header byte 20 */
    int32_t dt_us;       /* binary header byte 16 */
    double dt_seconds;
    int32_t format;      /* 1 IBM or 5 IEEE (unknown codes read as 5) */
    int32_t n_il, n_xl;  /* sorted unique INLINE_3D / CROSSLINE_3D labels (0 skipped) */
    int64_t n_mapped;    /* traces in the lookup table */
} psm_segy_info;

int psm_segy_scan(const char *path, psm_segy_info *info, char *err, size_t err_len);
/* Labels and the dense cube [n_il][n_xl][num_samples] (missing traces zero). */
int psm_segy_read_cube(const char *path, int32_t *il_labels, int32_t *xl_labels, float *cube,
                       char *err, size_t err_len);

/* IBM <-> IEEE single (src/segy_utils.cpp:243-270).  psm_ieee_to_ibm maps +-inf to the
 * largest IBM magnitude and NaN to 0x40000000 (the reference does not return on inf). */
float psm_ibm_to_ieee(uint32_t ibm);
uint32_t psm_ieee_to_ibm(float v);

/* Dense Vrms [n_il][n_xl][n_t] from a velocity parameter (number, .sgy/.segy path or text
 * table) on the given labels, as main.cpp:312-321 asks the provider per inline. */
int psm_velocity_cube(const char *param, const int32_t *il_labels, int32_t n_il,
                      const int32_t *xl_labels, int32_t n_xl, int32_t n_t, double dt,
                      float *out, char *err, size_t err_len);
/* VelocityProvider::getVelocity for one sample. */
int psm_velocity_point(const char *param, int32_t il, int32_t xl, int32_t t_idx, double dt,
                       int32_t n_t, float *out, char *err, size_t err_len);

/* Migration plan of a config (src/main.cpp:124-217): sizes, m_il, tan^2, estimated Vmax. */
typedef struct {
    int32_t n_il, n_xl, n_t;
    int32_t n_oi, n_ox;
    int32_t m_il;
    float max_v;
    float tan2_theta;
    double dt_seconds;
} psm_plan;
int psm_plan_config(const char *config_path, psm_plan *plan, char *err, size_t err_len);

/* The whole migration of a config file: read, migrate on the GPU, write the output SEG-Y
 * (src/main.cpp:66-442).  verbose prints the reference's progress lines on stdout. */
int psm_run_config(const char *config_path, int verbose, char *err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* PSM_HOST_H */
