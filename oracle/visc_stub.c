/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * Hydro/mhd.c defines no visc_source, but misc.c:571-573 calls it (behind
 * `if(visc_flag)`), so every cylindrical MHD build of the reference fails to
 * link as shipped.  Viscosity is off (Use_Viscosity 0) in every MHD config
 * here, so the call is never reached; this no-op only satisfies the linker.
 */
void visc_source(const double *prim, const double *gradr, const double *gradp,
                 const double *gradz, double *cons, const double *xp,
                 const double *xm, double dVdt){
   (void)prim; (void)gradr; (void)gradp; (void)gradz;
   (void)cons; (void)xp; (void)xm; (void)dVdt;
}
