/* Spectral sizes in the layout of RadChan's src/param/NarrowBand.h. */
#if grey == 0
#define nT 64
#define nQ 8
#define nB 100
#else
#define nT 65
#define nQ 1
#define nB 1000
#define abscoeff 1.f
#define Tmins 490.f
#define wvmax 5000.f
#endif
