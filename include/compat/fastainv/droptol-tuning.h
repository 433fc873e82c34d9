/* Drop-in for fastainv/droptol-tuning.h (reference
 * fastainv/droptol-tuning.h:4-103): DroptolTuner over the
 * ispm_droptol_tuner_* entry points -- the same droptol sequence for the same
 * reported times.  getBestDroptol() before the first noteTime() returns the
 * first probe (the reference leaves it undefined).  A tuner owns its search
 * state and cannot be copied. */
#ifndef FASTAINV_DROPTOL_TUNER_H
#define FASTAINV_DROPTOL_TUNER_H

#include "ispm_compat_detail.h"

class DroptolTuner {
  ispm_c::ispm_droptol_tuner *t;

 public:
  DroptolTuner(double lo = -10, double hi = -3) : t(ispm_c::ispm_droptol_tuner_create(lo, hi))
  {
    if (!t)
      ispm_compat::check(ISPM_ERR_NOMEM, "DroptolTuner");
  }
  ~DroptolTuner() { ispm_c::ispm_droptol_tuner_free(t); }
  DroptolTuner(const DroptolTuner &) = delete;
  DroptolTuner &operator=(const DroptolTuner &) = delete;

  double getDroptol() { return ispm_c::ispm_droptol_tuner_get_droptol(t); }
  double getBestDroptol() { return ispm_c::ispm_droptol_tuner_get_best_droptol(t); }
  void noteTime(double time) { ispm_c::ispm_droptol_tuner_note_time(t, time); }
  void restart() { ispm_c::ispm_droptol_tuner_restart(t); }
  void resetPhase() { ispm_c::ispm_droptol_tuner_reset_phase(t); }
  int iterations() { return ispm_c::ispm_droptol_tuner_iterations(t); }
};

#endif
