// subint.h -- division of time into sub-integrations: TimeDivide
// (Signal/Pulsar/TimeDivide.C) and the per-block loop of Subint<Fold>
// (Signal/Pulsar/dsp/Subint.h:258-332), with the MJD arithmetic they use.
#pragma once
#include <cstdint>
#include <vector>

namespace b200
{

// An epoch as whole days, whole seconds and a fraction of a second, kept
// normalised (0 <= sec < 86400, 0 <= frac < 1) as PSRCHIVE's MJD keeps it.
struct Mjd
{
  int64_t day = 0;
  int64_t sec = 0;
  double frac = 0.0;
};

Mjd mjd_add (const Mjd& a, double seconds);
double mjd_seconds_between (const Mjd& a, const Mjd& b);   // (a - b).in_seconds()
bool mjd_less (const Mjd& a, const Mjd& b);
bool mjd_equal (const Mjd& a, const Mjd& b);
inline bool mjd_is_zero (const Mjd& a) { return a.day == 0 && a.sec == 0 && a.frac == 0.0; }

// TimeDivide with a division length in seconds, or in turns of a constant
// folding period (the reference's branch without a Pulsar::Predictor).
class TimeDivide
{
public:
  double division_seconds = 0;
  double division_turns = 0;
  double period = 0;
  Mjd reference_epoch;          // zero: divisions start at the first data

  Mjd start_time;               // zero until the first block sets it

  // results of set_bounds
  bool is_valid = false, in_next = false, end_reached = false, new_division = false;
  uint64_t idat_start = 0, ndat = 0, division_ndat = 0, division = 0;
  Mjd lower, upper;

  void set_start_time (const Mjd& t);
  // set_bounds for an input of ndat samples at rate starting at start;
  // returns false (with *err set) where the reference throws
  bool set_bounds (const Mjd& start, uint64_t input_ndat, double rate, const char** err);

private:
  Mjd current_end;
  Mjd obs_start;
  double obs_rate = 0;
  bool set_boundaries (const Mjd& input_start, const char** err);
  void set_boundaries (const Mjd& mjd1, const Mjd& mjd2);
};

// One step of Subint<Fold>::transformation for a block: fold a range of the
// block's samples into the current sub-integration, or close (unload) it.
struct SubintAction
{
  enum Kind { FOLD = 0, CLOSE_PARTIAL = 1, CLOSE_COMPLETE = 2 };
  int kind = FOLD;
  bool end_reached = false;            // FOLD: the range ends its division
  uint64_t idat_start = 0, ndat = 0;   // FOLD: samples of the block
  uint64_t division = 0;
  Mjd lower, upper;                    // FOLD: the division's bounds
};

class SubintPlanner
{
public:
  TimeDivide divider;
  // the actions for one block (Subint::transformation); false on error
  bool block (const Mjd& start, uint64_t ndat, double rate, std::vector<SubintAction>* out,
              const char** err);
};

} // namespace b200
