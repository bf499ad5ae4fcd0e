/*
 * gf_footprint.h -- exact inside tests of the footprint regions (GF_FOOT_REGIONS),
 * shared by the host pixelisation and the device clipper.
 *
 * A region is one footprint specification of the reference (footprint.cpp:
 * load_footprint_beam :675-704 with makeBeamMap :591-673, load_footprint_rect
 * :486-589, clip_zone_of_avoidance :706-727, the union of the listed files in
 * load_footprints :746-758): a beam
 * (cap minus a concentric hole) or a lon/lat rectangle in galactic or equatorial
 * coordinates, minus the galactic band |b| < bmin.  Points are tested on the
 * sphere in double precision with the portable functions of gf_math.h.
 */
#pragma once
#include "../../include/galfast_b200.h"
#include "gf_math.h"

#if defined(__CUDACC__)
#define GFF_HD __host__ __device__ __forceinline__
#else
#define GFF_HD static inline
#endif

namespace gff {

/* galactic -> equatorial (J2000) unit vectors: the transpose of the ICRS-to-galactic
 * rotation of the Hipparcos catalogue (ESA 1997, vol. 1, section 1.5.3) */
GFF_HD void gal_to_equ(double l, double b, double &ra, double &dec)
{
    const double A[9] = {-0.0548755604162154, -0.8734370902348850, -0.4838350155487132,
                         +0.4941094278755837, -0.4448296299600112, +0.7469822444972189,
                         -0.8676661490190047, -0.1980763734312015, +0.4559837761750669};
    const double cb = gfm::cos_d(b);
    const double g[3] = {cb * gfm::cos_d(l), cb * gfm::sin_d(l), gfm::sin_d(b)};
    double e[3];
    for (int i = 0; i < 3; i++) e[i] = A[i] * g[0] + A[3 + i] * g[1] + A[6 + i] * g[2];
    ra = gfm::atan2_d(e[1], e[0]);
    double z = e[2];
    if (z > 1.0) z = 1.0;
    if (z < -1.0) z = -1.0;
    dec = gfm::asin_d(z);
}

/* equatorial (J2000) -> galactic, the inverse of gal_to_equ */
GFF_HD void equ_to_gal(double ra, double dec, double &l, double &b)
{
    const double A[9] = {-0.0548755604162154, -0.8734370902348850, -0.4838350155487132,
                         +0.4941094278755837, -0.4448296299600112, +0.7469822444972189,
                         -0.8676661490190047, -0.1980763734312015, +0.4559837761750669};
    const double cd = gfm::cos_d(dec);
    const double e[3] = {cd * gfm::cos_d(ra), cd * gfm::sin_d(ra), gfm::sin_d(dec)};
    double g[3];
    for (int i = 0; i < 3; i++) g[i] = A[3 * i] * e[0] + A[3 * i + 1] * e[1] + A[3 * i + 2] * e[2];
    l = gfm::atan2_d(g[1], g[0]);
    double z = g[2];
    if (z > 1.0) z = 1.0;
    if (z < -1.0) z = -1.0;
    b = gfm::asin_d(z);
}

/* is the galactic point (l, b) (degrees) inside region r? */
GFF_HD bool region_inside(const gf_region &r, double l, double b)
{
    const double d2r = 0.01745329251994329576923691;
    if (r.bmin > 0.0 && fabs(b) < r.bmin) return false;
    double lon = l * d2r, lat = b * d2r;
    if (r.coordsys == GF_COORD_EQU) gal_to_equ(lon, lat, lon, lat);
    if (r.type == GF_REGION_BEAM) {
        const double l0 = r.a * d2r, b0 = r.b * d2r;
        const double cosd = gfm::sin_d(lat) * gfm::sin_d(b0) + gfm::cos_d(lat) * gfm::cos_d(b0) * gfm::cos_d(lon - l0);
        if (r.c < 180.0 && !(cosd >= gfm::cos_d(r.c * d2r))) return false;
        if (r.d > 0.0 && cosd > gfm::cos_d(r.d * d2r)) return false;
        return true;
    }
    if (r.type == GF_REGION_RECT) {
        const double latd = lat / d2r;
        if (!(latd >= r.c && latd < r.d)) return false;
        if (r.a == r.b) return true;                       /* a full band of latitude */
        double lond = fmod(lon / d2r, 360.0);
        if (lond < 0) lond += 360.0;
        double a = fmod(r.a, 360.0), e = fmod(r.b, 360.0);
        if (a < 0) a += 360.0;
        if (e < 0) e += 360.0;
        return (a <= e) ? (lond >= a && lond < e) : (lond >= a || lond < e);
    }
    return false;
}

GFF_HD bool regions_inside(const gf_footprint &f, double l, double b)
{
    for (int i = 0; i < f.nregions && i < GF_MAX_REGIONS; i++)
        if (region_inside(f.regions[i], l, b)) return true;
    return false;
}

}  // namespace gff
