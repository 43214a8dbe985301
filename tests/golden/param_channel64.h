/* Parameter header in the layout of RadChan's src/param/param.h, for the
 * 64^3 narrow-band channel: three multigrid levels, adiabatic west wall. */
#define  num_gpu    1
#define  p_col      1
#define  imax       64
#define  jmax       64
#define  kmax       64
#define  Lx         2.f
#define  Ly         6.283185307179586f
#define  Lz         3.141592653589793f
#define  fact_mesh  1.5
#define  nVar       4
#define  photmax    256
#define  chanHeight 1.0

#define grid_num 3

const int maxi[] = {imax, imax/2, imax/4};
const int maxj[] = {jmax, jmax/2, jmax/4};
const int maxk[] = {kmax, kmax/2, kmax/4};
#if grid_num==1
const int maxs[] = {100000};
#elif grid_num==2
const int maxs[] = {5, 100000};
#elif grid_num==3
const int maxs[] = {5, 5, 100000};
#endif

#define num_streams     2
#define blockdim        128
#define nblocks         4096
#define srt 1
#define grey 0
#define calcwalls 1
#define random 0
#define floatpoint 0

#define  epsw   1.f
#define  epse   1.f
#define  epss   1.f
#define  epsn   1.f
#define  epsb   1.f
#define  epst   1.f
#define  Tww    955
#define  Twe    573
#define  Tws    0
#define  Twn    0
#define  Twb    0
#define  Twt    0
#define  adiabw 1
#define  adiabe 0
#define  stefan 5.670373e-08
#define  toll   1.0e-3
#define  tollS  1.0e-3
#define  pi     3.14159265358979323846
#define bdw 2
#define bde 2
#define bds 1
#define bdn 1
#define bdb 1
#define bdt 1

#if adiabw==1
#define boundini 0
#else
#define boundini 1
#endif
