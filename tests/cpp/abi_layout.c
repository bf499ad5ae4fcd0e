/* Prints the size of every C ABI struct and the offset of each field, one
 * "struct field offset" line per field ("struct - size" for the size), for the
 * test that compares them with the ctypes mirrors. */
#include <stddef.h>
#include <stdio.h>
#include "galfast_b200.h"

#define SZ(T) printf(#T " - %zu\n", sizeof(T))
#define OF(T, f) printf(#T " " #f " %zu\n", offsetof(T, f))

int main(void)
{
    SZ(gf_pencil_beam); OF(gf_pencil_beam, coveredFraction); OF(gf_pencil_beam, projIdx); OF(gf_pencil_beam, extIdx);
    SZ(gf_lambert); OF(gf_lambert, cl);
    SZ(gf_skygen_config); OF(gf_skygen_config, nthreads); OF(gf_skygen_config, nstars); OF(gf_skygen_config, proj);
    SZ(gf_model_config); OF(gf_model_config, f); OF(gf_model_config, frame); OF(gf_model_config, Rg); OF(gf_model_config, M);
    OF(gf_model_config, lf_l); OF(gf_model_config, lf_M); OF(gf_model_config, lf_n); OF(gf_model_config, nbreaks);
    OF(gf_model_config, n_brk); OF(gf_model_config, rbreak); OF(gf_model_config, cube); OF(gf_model_config, cube_n);
    OF(gf_model_config, cube_tc);
    SZ(gf_ext_map); OF(gf_ext_map, n); OF(gf_ext_map, tc); OF(gf_extinction, north); OF(gf_extinction, south);
    SZ(gf_region); OF(gf_region, bmin); OF(gf_footprint, nregions); OF(gf_footprint, regions);
    SZ(gf_extinction); SZ(gf_footprint); OF(gf_footprint, a);
    SZ(gf_table); OF(gf_table, nbands); OF(gf_table, lb); OF(gf_table, hidden); OF(gf_table, radec); OF(gf_table, FeH_comp); OF(gf_table, absmagSysNcomp); OF(gf_table, systems);
    SZ(gf_fixedfeh_config); SZ(gf_vmoments); SZ(gf_bond2010_config); OF(gf_bond2010_config, halo); OF(gf_bond2010_config, T);
    SZ(gf_feh_config); OF(gf_feh_config, Hmu); OF(gf_feh_config, comp_thin); OF(gf_feh_config, M); OF(gf_feh_config, T);
    SZ(gf_gaussfeh_config); OF(gf_gaussfeh_config, sigma); OF(gf_gaussfeh_config, comp_mask);
    SZ(gf_photometry_config); OF(gf_photometry_config, reddening); OF(gf_photometry_config, nFeH); OF(gf_photometry_config, colors);
    OF(gf_photometry_config, comp_mask);
    SZ(gf_photoerr_config); OF(gf_photoerr_config, mag); OF(gf_photoerr_config, seed);
    SZ(gf_vel2pm_config); OF(gf_vel2pm_config, Rg);
    SZ(gf_skygen_model_info); OF(gf_skygen_model_info, nm); OF(gf_skygen_model_info, norm);
    SZ(gf_job); OF(gf_job, pixels); OF(gf_job, ext); OF(gf_job, models); OF(gf_job, seed48); OF(gf_job, capacity);
    OF(gf_job, foot); OF(gf_job, v2pm); OF(gf_job, gal2other); OF(gf_job, feh_ivezic); OF(gf_job, feh_gauss); OF(gf_job, multiples);
    SZ(gf_catalog_stats); OF(gf_catalog_stats, generated); OF(gf_catalog_stats, batches); OF(gf_catalog_stats, norm);
    SZ(gf_precision_report); OF(gf_precision_report, bins);
    SZ(gf_textout_config); OF(gf_textout_config, nbands); OF(gf_textout_config, feh_comp); OF(gf_textout_config, comp_ids);
    OF(gf_textout_config, version); OF(gf_textout_config, threads); OF(gf_textout_config, multiples);
    SZ(gf_multiples_config); OF(gf_multiples_config, nsec); OF(gf_multiples_config, cumlf); OF(gf_multiples_config, ninv);
    OF(gf_multiples_config, invcumlf);
    SZ(gf_textout_set); OF(gf_textout_set, writers);
    SZ(gf_server_info); OF(gf_server_info, deferred); OF(gf_server_info, peak_running); OF(gf_server_info, active);
    return 0;
}
