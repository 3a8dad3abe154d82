// geom.h — epochs, source coordinates and the baseline geometric delay model
// feeding the 1-s delay table (fx-corr src/geom.rs).
#pragma once

#include <cstdint>
#include <string>

namespace yi {

constexpr double kYamagu32Ecef[3] = {-3502544.587, 3950966.235, 3566381.192};  // geom.rs:7
constexpr double kYamagu34Ecef[3] = {-3502567.576, 3950885.734, 3566449.115};  // geom.rs:8

// RA / Dec strings to radians (geom.rs:87-151): h/m/s or d/m/s markers, colons,
// packed hhmmss / ddmmss, or decimal degrees.  Throw std::runtime_error.
double parse_ra(const std::string& s);
double parse_dec(const std::string& s);
// Epoch to MJD (geom.rs:153-269): ISO 8601, YYYY/DDD [HH:MM:SS], MJD, or a
// (J-prefixed) year.
double parse_epoch_to_mjd(const std::string& s);
// cor.rs:299-306
int64_t mjd_to_unix_seconds(double mjd);
int64_t epoch_to_unix_seconds(const std::string& s);

// Greenwich sidereal time (rad, [0, 2 pi)) with UT1 = TT = UTC as the reference
// assumes (geom.rs:289-294): mean sidereal time from the Earth rotation angle
// and the IAU 2006 GMST polynomial (IERS Conventions 2010, eqs. 5.15 and 5.32);
// apparent adds the equation of the equinoxes from the abridged nutation of
// Meeus, Astronomical Algorithms, ch. 22 (about 0.5 arcsec).
double gmst_rad(double mjd);
double gast_rad(double mjd);

// J2000 mean RA/Dec to mean equator and equinox of date (geom.rs:278-285),
// by the IAU 1976 precession angles zeta, z, theta (Lieske et al. 1977) in the
// rigorous form of Meeus ch. 21.
void precess_j2000_to_mean_of_date(double ra, double dec, double mjd, double* ra_d,
                                   double* dec_d);

// (delay ant1, delay ant2, baseline delay, rate, accel) (geom.rs:353-385):
// tau = -(B . s)/c with B = ant2 - ant1, derivatives by central differences
// over +-1 s.
struct GeomDelay {
  double delay1, delay2, delay, rate, accel;
};
GeomDelay geometric_delay_and_derivatives(const double ant1[3], const double ant2[3], double ra,
                                          double dec, double mjd);
double baseline_delay(const double ant1[3], const double ant2[3], double ra, double dec,
                      double mjd);

}  // namespace yi
