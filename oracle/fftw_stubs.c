/*
 * Abort-stubs for the four reference functions whose sources need FFTW
 * (not installed here).  None of them is on the P-SV forward / L2-gradient
 * path (envelope misfits, Hilbert transforms, source-wavelet inversion and
 * wavenumber filtering are all switched off in the oracle's parameter files);
 * they exist only so the reference binary links.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>

static void dn_oracle_no_fftw(const char *name)
{
    fprintf(stderr, "oracle build: %s needs FFTW, which this build leaves out\n", name);
    exit(3);
}

void calc_envelope(float **datatrace, float **envelope, int ns, int ntr)
{ (void)datatrace; (void)envelope; (void)ns; (void)ntr; dn_oracle_no_fftw("calc_envelope"); }

void calc_hilbert(float **datatrace, float **envelope, int ns, int ntr)
{ (void)datatrace; (void)envelope; (void)ns; (void)ntr; dn_oracle_no_fftw("calc_hilbert"); }

void conv_FD(float *temp_TS, float *temp_TS1, float *temp_conv, int ns)
{ (void)temp_TS; (void)temp_TS1; (void)temp_conv; (void)ns; dn_oracle_no_fftw("conv_FD"); }

void stf(float **sectionvy_obs, float **sectionvy, int ntr_glob, int ishot, int ns, int iter, int nshots,
         float **signals, int **recpos, float **srcpos)
{
    (void)sectionvy_obs; (void)sectionvy; (void)ntr_glob; (void)ishot; (void)ns; (void)iter; (void)nshots;
    (void)signals; (void)recpos; (void)srcpos;
    dn_oracle_no_fftw("stf");
}

void wavenumber(float **grad) { (void)grad; dn_oracle_no_fftw("wavenumber"); }
