// Drop-tolerance search by golden-section steps over log2(droptol)
// (the DroptolTuner interface of fastainv/droptol-tuning.h:4-103).
//
// State: a bracket end[0] < end[1] and two interior probes p[0] < p[1]
// placed symmetrically in it (p[0] = end0 + (end1 - end0) * (2 - phi),
// p[1] = end0 + (end1 - p[0])).  The caller solves with the droptol of the
// probe handed out (slot `next`) and reports the time.  Once both probes are
// timed, the slower probe becomes the new bracket end on its side, the
// faster probe moves into the vacated slot and a new probe is mirrored into
// its old one: the only untimed probe, so it is the next one handed out.  The
// first report after construction, restart() or reset_phase() times p[0]
// only and restarts the record of the best droptol.
//
// Callers see the reference's droptol sequence: the placement and mirroring
// are the same arithmetic, and the bracket always keeps the side of the
// strictly faster probe (ties keep the upper side).
#include <cmath>
#include <limits>
#include <new>

#include "ispm_internal.h"

namespace {

constexpr double kGolden = .3819660112501051518;  // 2 - phi: the short section

struct GoldenBracket {
  double end[2];       // bracket ends, log2 droptol
  double p[2];         // interior probes
  double t[2] = {0, 0};// solve times measured at the probes
  int next = 0;        // probe handed out next
  bool opening = true; // the next report is the first of a (re)started search
  double best_x;
  double best_t = std::numeric_limits<double>::infinity();
  int steps = 0;       // bracket reductions since construction / restart()

  GoldenBracket(double lo, double hi)
  {
    place(lo, hi);
    best_x = p[0];
  }

  void place(double lo, double hi)
  {
    end[0] = lo;
    end[1] = hi;
    p[0] = lo + (hi - lo) * kGolden;
    p[1] = mirror(p[0]);
  }
  double mirror(double q) const { return end[0] + (end[1] - q); }

  void report(double time)
  {
    if (opening || best_t > time) {
      best_t = time;
      best_x = p[next];
    }
    t[next] = time;
    if (opening) {  // one side timed: hand out the other probe
      opening = false;
      next = 1;
      return;
    }
    const int keep = t[0] < t[1] ? 0 : 1, drop = 1 - keep;
    end[drop] = p[drop];
    p[drop] = p[keep];
    t[drop] = t[keep];
    p[keep] = mirror(p[drop]);
    next = keep;
    steps++;
  }

  // A narrower search (+-1 in log2) around the lower probe.
  void restart()
  {
    const double c = p[0];
    place(c - 1, c + 1);
    next = 0;
    opening = true;
    steps = 0;
  }
  void reset_phase()
  {
    next = 0;
    opening = true;
  }
};

}  // namespace

struct ispm_droptol_tuner {
  GoldenBracket g;
};

extern "C" {

ispm_droptol_tuner *ispm_droptol_tuner_create(double lo, double hi)
{
  return new (std::nothrow) ispm_droptol_tuner{GoldenBracket(lo, hi)};
}
double ispm_droptol_tuner_get_droptol(const ispm_droptol_tuner *t)
{
  return std::exp2(t->g.p[t->g.next]);
}
double ispm_droptol_tuner_get_best_droptol(const ispm_droptol_tuner *t)
{
  return std::exp2(t->g.best_x);
}
void ispm_droptol_tuner_note_time(ispm_droptol_tuner *t, double time) { t->g.report(time); }
void ispm_droptol_tuner_restart(ispm_droptol_tuner *t) { t->g.restart(); }
void ispm_droptol_tuner_reset_phase(ispm_droptol_tuner *t) { t->g.reset_phase(); }
int ispm_droptol_tuner_iterations(const ispm_droptol_tuner *t) { return t->g.steps; }
void ispm_droptol_tuner_free(ispm_droptol_tuner *t) { delete t; }

}  // extern "C"
