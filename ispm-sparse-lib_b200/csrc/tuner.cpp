// Golden-section drop-tolerance tuner (fastainv/droptol-tuning.h:4-103).
//
// The search runs over log2(droptol): each noteTime() reports the solve time
// measured with the droptol last handed out, and the bracket shrinks by the
// golden ratio towards the faster side.  The probe sequence is the
// reference's, so a caller swapping implementations sees the same droptols.
#include <cmath>
#include <limits>
#include <new>

#include "ispm_internal.h"

namespace {

class DroptolTuner {
  enum Phase { kFirstM1, kM1, kM2 };
  static constexpr double kRatio = .3819660112501051518;  // 2 - golden ratio

  static double left(double lo, double hi) { return lo + (hi - lo) * kRatio; }
  static double mirror(double lo, double hi, double mid) { return lo + (hi - mid); }

  Phase phase_;
  double lo_, hi_, m1_, m2_, best_;
  double t1_ = 0, t2_ = 0, tbest_;
  int iters_ = 0;

 public:
  DroptolTuner(double lo, double hi)
      : phase_(kFirstM1), lo_(lo), hi_(hi), m1_(left(lo, hi)), m2_(mirror(lo, hi, m1_)),
        best_(m1_), tbest_(std::numeric_limits<double>::infinity())
  {
  }
  double droptol() const { return std::exp2(phase_ == kM2 ? m2_ : m1_); }
  double best() const { return std::exp2(best_); }
  int iterations() const { return iters_; }
  void reset_phase() { phase_ = kFirstM1; }
  void restart()
  {
    phase_ = kFirstM1;
    lo_ = m1_ - 1;
    hi_ = m1_ + 1;
    m1_ = left(lo_, hi_);
    m2_ = mirror(lo_, hi_, m1_);
    iters_ = 0;
  }
  void note(double time)
  {
    switch (phase_) {
    case kFirstM1:
      tbest_ = time;
      best_ = m1_;
      t1_ = time;
      phase_ = kM2;
      return;
    case kM2:
      if (tbest_ > time) {
        tbest_ = time;
        best_ = m2_;
      }
      t2_ = time;
      break;
    case kM1:
      if (tbest_ > time) {
        tbest_ = time;
        best_ = m1_;
      }
      t1_ = time;
      break;
    }
    if (t1_ < t2_) {
      hi_ = m2_;
      m2_ = m1_;
      m1_ = mirror(lo_, hi_, m2_);
      t2_ = t1_;
      phase_ = kM1;
    } else {
      lo_ = m1_;
      m1_ = m2_;
      m2_ = mirror(lo_, hi_, m1_);
      t1_ = t2_;
      phase_ = kM2;
    }
    iters_++;
  }
};

}  // namespace

struct ispm_droptol_tuner {
  DroptolTuner t;
};

extern "C" {

ispm_droptol_tuner *ispm_droptol_tuner_create(double lo, double hi)
{
  return new (std::nothrow) ispm_droptol_tuner{DroptolTuner(lo, hi)};
}
double ispm_droptol_tuner_get_droptol(const ispm_droptol_tuner *t) { return t->t.droptol(); }
double ispm_droptol_tuner_get_best_droptol(const ispm_droptol_tuner *t) { return t->t.best(); }
void ispm_droptol_tuner_note_time(ispm_droptol_tuner *t, double time) { t->t.note(time); }
void ispm_droptol_tuner_restart(ispm_droptol_tuner *t) { t->t.restart(); }
void ispm_droptol_tuner_reset_phase(ispm_droptol_tuner *t) { t->t.reset_phase(); }
int ispm_droptol_tuner_iterations(const ispm_droptol_tuner *t) { return t->t.iterations(); }
void ispm_droptol_tuner_free(ispm_droptol_tuner *t) { delete t; }

}  // extern "C"
