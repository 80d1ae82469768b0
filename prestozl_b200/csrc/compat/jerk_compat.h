/*
 * Shared by the drop-in's compat files: the search geometry of the
 * reference's accelobs (include/accel.h:43-82) as the plain jerk_obs of
 * jerk.h.  Include it after the reference's accel.h (which has no include
 * guard, so it is not included again here) and jerk.h.
 */
#ifndef JERK_COMPAT_H
#define JERK_COMPAT_H

#include <string.h>

static inline void jerk_obs_of_accelobs(const accelobs *obs, jerk_obs *o)
{
    memset(o, 0, sizeof(*o));
    o->numbins = obs->numbins;
    o->lobin = obs->lobin;
    o->highestbin = obs->highestbin;
    o->rlo = obs->rlo;
    o->zlo = obs->zlo;
    o->wlo = obs->wlo;
    o->corr_uselen = obs->corr_uselen;
    o->numz = obs->numz;
    o->numw = obs->numw;
    o->numharmstages = obs->numharmstages;
    o->norm_type = obs->norm_type;
    o->nph = obs->nph;
    for (int ii = 0; ii < obs->numharmstages && ii < JERK_MAX_STAGES; ii++) {
        o->powcut[ii] = obs->powcut[ii];
        o->numindep[ii] = obs->numindep[ii];
    }
}

#endif
