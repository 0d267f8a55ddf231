// subint.cpp -- TimeDivide (Signal/Pulsar/TimeDivide.C) and the block loop of
// Subint<Fold> (Signal/Pulsar/dsp/Subint.h:258-332), restated for the fused
// pipeline, which folds every range of a block in one pass.
#include "subint.h"

#include <cmath>

namespace b200
{

Mjd mjd_add (const Mjd& a, double seconds)
{
  Mjd r = a;
  const double f = a.frac + seconds;
  const double whole = std::floor (f);
  r.frac = f - whole;
  int64_t s = a.sec + int64_t (whole);
  int64_t d = s / 86400;
  s -= d * 86400;
  if (s < 0) { s += 86400; d -= 1; }
  r.sec = s;
  r.day = a.day + d;
  return r;
}

double mjd_seconds_between (const Mjd& a, const Mjd& b)
{
  return double ((a.day - b.day) * 86400 + (a.sec - b.sec)) + (a.frac - b.frac);
}

bool mjd_less (const Mjd& a, const Mjd& b)
{
  if (a.day != b.day) return a.day < b.day;
  if (a.sec != b.sec) return a.sec < b.sec;
  return a.frac < b.frac;
}

bool mjd_equal (const Mjd& a, const Mjd& b)
{
  return a.day == b.day && a.sec == b.sec && a.frac == b.frac;
}

static const Mjd& mjd_max (const Mjd& a, const Mjd& b) { return mjd_less (a, b) ? b : a; }
static const Mjd& mjd_min (const Mjd& a, const Mjd& b) { return mjd_less (b, a) ? b : a; }

// TimeDivide::set_start_time (TimeDivide.C:40-76): a reference epoch wins;
// else an integer division length in seconds aligns the start to a multiple
// of it within the day
void TimeDivide::set_start_time (const Mjd& t)
{
  if (mjd_equal (start_time, t))
    return;
  start_time = t;
  is_valid = false;
  if (!mjd_is_zero (reference_epoch))
    start_time = reference_epoch;
  else if (division_seconds != 0 && division_seconds == double (unsigned (division_seconds)))
  {
    const unsigned integer_seconds = unsigned (division_seconds);
    const unsigned seconds = unsigned (start_time.sec);
    const unsigned divisions = seconds / integer_seconds;
    start_time.sec = int64_t (divisions) * integer_seconds;
    start_time.frac = 0.0;
  }
}

// TimeDivide::set_boundaries (const MJD&, const MJD&) (TimeDivide.C:503-537):
// the bounds rounded to whole samples of the current input
void TimeDivide::set_boundaries (const Mjd& mjd1, const Mjd& mjd2)
{
  double seconds = mjd_seconds_between (mjd1, obs_start);
  const int64_t samples = std::lrint (seconds * obs_rate);
  lower = mjd_add (obs_start, double (samples) / obs_rate);
  seconds = mjd_seconds_between (mjd2, lower);
  division_ndat = uint64_t (std::lrint (seconds * obs_rate));
  upper = mjd_add (lower, double (division_ndat) / obs_rate);
}

// TimeDivide::set_boundaries (const MJD&) (TimeDivide.C:349-501), the branch
// of a division length in seconds or in turns of a constant period
bool TimeDivide::set_boundaries (const Mjd& input_start, const char** err)
{
  if (mjd_is_zero (start_time))
  {
    *err = "TimeDivide: observation start time not set";
    return false;
  }
  const Mjd& divide_start = mjd_max (start_time, input_start);
  if (!(division_seconds > 0 || (division_turns != 0 && period > 0.0)))
  {
    *err = "TimeDivide: division length not specified (seconds, or turns with a period)";
    return false;
  }
  const double seconds = mjd_seconds_between (divide_start, start_time);
  double seconds_per_interval = division_seconds;
  if (division_turns != 0)
    seconds_per_interval = period * division_turns;
  division = uint64_t (seconds / seconds_per_interval);
  set_boundaries (mjd_add (start_time, double (division) * seconds_per_interval),
                  mjd_add (start_time, double (division + 1) * seconds_per_interval));
  return true;
}

// TimeDivide::set_bounds (TimeDivide.C:130-333)
bool TimeDivide::set_bounds (const Mjd& input_start, uint64_t input_ndat, double rate,
                             const char** err)
{
  obs_start = input_start;
  obs_rate = rate;
  const Mjd input_end = input_ndat ? mjd_add (input_start, double (input_ndat) / rate)
                                   : input_start;
  Mjd divide_start = input_start;
  if (is_valid)
    divide_start = mjd_max (current_end, input_start);
  new_division = false;
  end_reached = false;
  in_next = false;
  if (mjd_less (input_end, lower) || mjd_less (upper, mjd_add (divide_start, 0.5 / rate)))
  {
    new_division = true;
    if (!set_boundaries (mjd_add (divide_start, 0.55 / rate), err))
      return false;
  }
  divide_start = mjd_max (lower, divide_start);

  const double start_sample = std::rint (mjd_seconds_between (divide_start, input_start) * rate);
  if (start_sample < 0)
  {
    *err = "TimeDivide: start sample before the input";
    return false;
  }
  idat_start = uint64_t (start_sample);
  if (idat_start >= input_ndat)
  {
    is_valid = false;
    return true;
  }
  const Mjd& divide_end = mjd_min (input_end, upper);
  const double end_sample = std::rint (mjd_seconds_between (divide_end, input_start) * rate);
  uint64_t idat_end = end_sample > 0 ? uint64_t (end_sample) : 0;
  if (idat_end <= idat_start)
  {
    *err = "TimeDivide: idat_end <= idat_start";
    return false;
  }
  if (idat_end > input_ndat)
    idat_end = input_ndat;                // rounding in rint
  else if (idat_end < input_ndat)
    in_next = true;                       // the input reaches the next division
  ndat = idat_end - idat_start;
  const double samples_to_end = mjd_seconds_between (upper, divide_end) * rate;
  if (samples_to_end < 0.5)
    end_reached = true;
  is_valid = true;
  current_end = mjd_add (input_start, double (idat_end) / rate);
  return true;
}

// Subint<Fold>::prepare (Subint.h:206-245) and transformation (:248-332)
bool SubintPlanner::block (const Mjd& start, uint64_t ndat, double rate,
                           std::vector<SubintAction>* out, const char** err)
{
  out->clear ();
  if (mjd_is_zero (divider.start_time))
  {
    if (mjd_is_zero (start))
    {
      *err = "Subint: input start time not set";
      return false;
    }
    divider.set_start_time (start);
  }
  bool more = true, first = true;
  // each pass ends one division inside the block: a block of ndat samples
  // cannot take more than ndat + 2 passes
  for (uint64_t guard = 0; more; guard++)
  {
    if (guard > ndat + 2)
    {
      *err = "Subint: division of the block does not advance";
      return false;
    }
    if (!divider.set_bounds (start, ndat, rate, err))
      return false;
    more = divider.in_next;
    SubintAction a;
    if (first && divider.new_division)
    {
      a.kind = SubintAction::CLOSE_PARTIAL;
      out->push_back (a);
    }
    if (!divider.is_valid)
      continue;
    a.kind = SubintAction::FOLD;
    a.idat_start = divider.idat_start;
    a.ndat = divider.ndat;
    a.division = divider.division;
    a.lower = divider.lower;
    a.upper = divider.upper;
    a.end_reached = divider.end_reached;
    out->push_back (a);
    if (!divider.end_reached)
      continue;
    SubintAction c;
    if (first)
    {
      c.kind = SubintAction::CLOSE_PARTIAL;
      out->push_back (c);
      first = false;
      continue;
    }
    c.kind = SubintAction::CLOSE_COMPLETE;
    out->push_back (c);
  }
  return true;
}

} // namespace b200

// ---------------------------------------------------------------------------
// C ABI: the division of time on its own (host only)
// ---------------------------------------------------------------------------

#include "dada.h"

struct dspsr_b200_time_divide
{
  b200::SubintPlanner planner;
  std::vector<b200::SubintAction> actions;
};

namespace
{
void to_action (const b200::SubintAction& a, dspsr_b200_subint_action* o)
{
  o->kind = a.kind;
  o->end_reached = a.end_reached ? 1 : 0;
  o->idat_start = a.idat_start;
  o->ndat = a.ndat;
  o->division = a.division;
  o->lower_day = a.lower.day;
  o->lower_sec = a.lower.sec;
  o->lower_frac = a.lower.frac;
  o->upper_day = a.upper.day;
  o->upper_sec = a.upper.sec;
  o->upper_frac = a.upper.frac;
}
}

extern "C" {

int dspsr_b200_time_divide_create (double seconds, double turns, double period_s,
                                   int64_t epoch_day, int64_t epoch_sec, double epoch_frac,
                                   dspsr_b200_time_divide** td)
{
  using dspsr_b200_host::host_fail;
  if (!td) return host_fail (DSPSR_B200_EINVAL, "time_divide_create: null output");
  *td = nullptr;
  if (!(seconds > 0) && !(turns > 0 && period_s > 0))
    return host_fail (DSPSR_B200_EINVAL,
                      "time_divide_create: seconds=%g, turns=%g, period=%g: give a division "
                      "length in seconds, or in turns with a period", seconds, turns, period_s);
  auto* t = new dspsr_b200_time_divide;
  b200::TimeDivide& d = t->planner.divider;
  // set_seconds / set_turns clear each other (TimeDivide.C:78-96)
  if (seconds > 0) d.division_seconds = seconds;
  else d.division_turns = turns;
  d.period = period_s;
  d.reference_epoch.day = epoch_day;
  d.reference_epoch.sec = epoch_sec;
  d.reference_epoch.frac = epoch_frac;
  *td = t;
  return DSPSR_B200_OK;
}

int dspsr_b200_time_divide_block (dspsr_b200_time_divide* td, int64_t start_day,
                                  int64_t start_sec, double start_frac, uint64_t ndat,
                                  double rate, dspsr_b200_subint_action* actions, uint64_t cap,
                                  uint64_t* n)
{
  using dspsr_b200_host::host_fail;
  if (!td || !n || (!actions && cap)) return host_fail (DSPSR_B200_EINVAL, "time_divide_block: null argument");
  *n = 0;
  if (!(rate > 0)) return host_fail (DSPSR_B200_EINVAL, "time_divide_block: rate=%g", rate);
  b200::Mjd s;
  s.day = start_day;
  s.sec = start_sec;
  s.frac = start_frac;
  const char* err = nullptr;
  if (!td->planner.block (s, ndat, rate, &td->actions, &err))
    return host_fail (DSPSR_B200_ESTATE, "%s", err);
  if (td->actions.size () > cap)
    return host_fail (DSPSR_B200_ETOOBIG, "time_divide_block: %llu actions, room for %llu",
                      (unsigned long long) td->actions.size (), (unsigned long long) cap);
  for (size_t i = 0; i < td->actions.size (); i++)
    to_action (td->actions[i], actions + i);
  *n = td->actions.size ();
  return DSPSR_B200_OK;
}

int dspsr_b200_time_divide_destroy (dspsr_b200_time_divide* td)
{
  if (!td) return DSPSR_B200_EINVAL;
  delete td;
  return DSPSR_B200_OK;
}

}  // extern "C"
