// dada.cpp -- the DADA file source of the hot path: the ASCII header rules
// (Kernel/Classes/ascii_header.c), DADAHeader::load_header / valid
// (Kernel/Classes/DADAHeader.C), the keys ASCIIObservation::load reads
// (Kernel/Classes/ASCIIObservation.C) and File's byte <-> sample arithmetic
// (Kernel/Classes/File.C).  Host code only: blocks read here go to the
// device through dspsr_b200_pipeline_run_dada (capi.cu).
#include "dada.h"
#include "subint.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

namespace dspsr_b200_host
{
thread_local std::string host_error;

int host_fail (int code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start (ap, fmt);
  vsnprintf (buf, sizeof (buf), fmt, ap);
  va_end (ap);
  host_error = buf;
  return code;
}
}  // namespace dspsr_b200_host

using dspsr_b200_host::host_fail;
using dspsr_b200_host::host_error;
using b200::mjd_add;

namespace
{

// DADAHeader::default_header_size (DADAHeader.C:22)
constexpr uint64_t DEFAULT_HEADER_SIZE = 4096;
// the reference scans string values into char[64]
constexpr size_t VALUE_MAX = 64;

bool is_space (char c)
{
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// ascii_header_find (ascii_header.c:34-56): the first occurrence of keyword
// that is the first word of the header, or that follows a newline or a
// backslash and is followed by a blank or a tab.
const char* header_find (const char* header, const char* keyword)
{
  const size_t len = strlen (keyword);
  const char* key = strstr (header, keyword);
  while (key && key > header)
  {
    const char before = key[-1];
    const char after = key[len];
    if ((before == '\n' || before == '\\') && (after == '\t' || after == ' '))
      break;
    key = strstr (key + 1, keyword);
  }
  return key;
}

// ascii_header_get with "%s" (ascii_header.c:117-142): the value starts at
// the first blank after the keyword's first byte; scanf skips white space and
// takes the next token.  Returns 1, or -1 for a missing keyword or an empty
// value (scanf's EOF).
int header_token (const char* header, const char* keyword, std::string& token)
{
  const char* key = header_find (header, keyword);
  if (!key)
    return -1;
  const char* v = key + strcspn (key, " \t\n");
  while (*v && is_space (*v))
    v++;
  if (!*v)
    return -1;
  const char* e = v;
  while (*e && !is_space (*e))
    e++;
  token.assign (v, e - v);
  return 1;
}

// The numeric scanf codes of ASCIIObservation::load: 1 when the token starts
// with a number, 0 when it does not (a scanf matching failure), -1 absent.
int header_double (const char* header, const char* keyword, double* out)
{
  std::string t;
  if (header_token (header, keyword, t) < 0)
    return -1;
  char* end = nullptr;
  const double v = strtod (t.c_str (), &end);
  if (end == t.c_str ())
    return 0;
  *out = v;
  return 1;
}

int header_int64 (const char* header, const char* keyword, int64_t* out)
{
  std::string t;
  if (header_token (header, keyword, t) < 0)
    return -1;
  char* end = nullptr;
  const long long v = strtoll (t.c_str (), &end, 10);
  if (end == t.c_str ())
    return 0;
  *out = v;
  return 1;
}

int header_uint64 (const char* header, const char* keyword, uint64_t* out)
{
  std::string t;
  if (header_token (header, keyword, t) < 0)
    return -1;
  char* end = nullptr;
  const unsigned long long v = strtoull (t.c_str (), &end, 10);
  if (end == t.c_str ())
    return 0;
  *out = v;
  return 1;
}

void copy_value (char* dst, const std::string& s)
{
  const size_t n = std::min (s.size (), VALUE_MAX - 1);
  memcpy (dst, s.data (), n);
  dst[n] = '\0';
}

// The MJD of a UTC date "YYYY-MM-DD-hh:mm:ss" (ASCIIObservation.C:322-340:
// strptime, then timegm seconds since 1970-01-01 = MJD 40587).
bool utc_to_mjd (const char* text, int64_t* day, int64_t* sec)
{
  struct tm utc;
  memset (&utc, 0, sizeof (utc));
  if (!strptime (text, "%Y-%m-%d-%H:%M:%S", &utc))
    return false;
  const int64_t t = int64_t (timegm (&utc));
  int64_t d = t / 86400, s = t % 86400;
  if (s < 0) { s += 86400; d -= 1; }
  *day = 40587 + d;
  *sec = s;
  return true;
}

// MJD += seconds on the info's (day, sec, frac) fields
void mjd_add (int64_t* day, int64_t* sec, double* frac, double seconds)
{
  b200::Mjd m;
  m.day = *day;
  m.sec = *sec;
  m.frac = *frac;
  m = b200::mjd_add (m, seconds);
  *day = m.day;
  *sec = m.sec;
  *frac = m.frac;
}

// replace_extension (psrchive's Util/genutil, used by DADAHeader.C:89): the
// text from the last '.' of the file name (not of a directory) is replaced,
// or the extension appended when the name has none.
std::string replace_extension (const std::string& name, const std::string& ext)
{
  const size_t slash = name.find_last_of ('/');
  const size_t dot = name.find_last_of ('.');
  if (dot == std::string::npos || (slash != std::string::npos && dot < slash))
    return name + ext;
  return name.substr (0, dot) + ext;
}

int read_file (const std::string& path, std::string& text, uint64_t nbyte, bool exact)
{
  FILE* f = fopen (path.c_str (), "rb");
  if (!f)
    return host_fail (DSPSR_B200_EINVAL, "fopen (%s): %s", path.c_str (), strerror (errno));
  text.assign (nbyte, '\0');
  const size_t got = fread (&text[0], 1, nbyte, f);
  fclose (f);
  if (exact && got != nbyte)
    return host_fail (DSPSR_B200_EINVAL, "fread (nbyte=%llu) of %s", (unsigned long long) nbyte,
                      path.c_str ());
  text.resize (nbyte);
  return DSPSR_B200_OK;
}

// DADAHeader::load_header (DADAHeader.C:56-139)
int load_header (const char* filename, std::string& header, uint64_t* hdr_size, int* adjacent)
{
  *adjacent = 0;
  uint64_t size = DEFAULT_HEADER_SIZE;
  uint64_t buffer = 0;
  do
  {
    buffer = size;
    int rc = read_file (filename, header, buffer, true);
    if (rc) return rc;
    header[buffer - 1] = '\0';
    uint64_t v = 0;
    size = header_uint64 (header.c_str (), "HDR_SIZE", &v) == 1 ? v : 0;
  }
  while (size > buffer);

  if (size == 0)
  {
    // an adjacent header file: name.hdr for name.ext, else name + ".hdr"
    std::string path = replace_extension (filename, ".hdr");
    struct stat st;
    if (stat (path.c_str (), &st) != 0)
    {
      path = std::string (filename) + ".hdr";
      if (stat (path.c_str (), &st) != 0)
        return host_fail (DSPSR_B200_EINVAL,
                          "%s: file has no header and no adjacent header file found", filename);
    }
    const uint64_t n = uint64_t (st.st_size);
    if (n == 0)
      return host_fail (DSPSR_B200_EINVAL, "%s: empty adjacent header file", path.c_str ());
    int rc = read_file (path, header, n, true);
    if (rc) return rc;
    header[n - 1] = '\0';
    *adjacent = 1;
    // HDR_SIZE in an adjacent header is a block of bytes to skip in the data
    uint64_t v = 0;
    size = header_uint64 (header.c_str (), "HDR_SIZE", &v) == 1 ? v : 0;
  }
  *hdr_size = size;
  return DSPSR_B200_OK;
}

}  // namespace

struct dspsr_b200_dada_file
{
  int fd = -1;
  std::string header;
  dspsr_b200_dada_info info;
  uint64_t data_end = 0;   // byte offset of the end of the data
};

extern "C" {

const char* dspsr_b200_host_error (void)
{
  return host_error.c_str ();
}

int dspsr_b200_ascii_header_get (const char* header, const char* keyword, char* value,
                                 uint64_t value_cap)
{
  if (!header || !keyword || !value || value_cap == 0)
    return host_fail (-1, "ascii_header_get: null argument");
  std::string t;
  if (header_token (header, keyword, t) < 0)
    return -1;
  const size_t n = std::min<uint64_t> (t.size (), value_cap - 1);
  memcpy (value, t.data (), n);
  value[n] = '\0';
  return 1;
}

int dspsr_b200_ascii_header_set (char* header, uint64_t header_cap, const char* keyword,
                                 const char* value)
{
  if (!header || !keyword || !value)
    return host_fail (DSPSR_B200_EINVAL, "ascii_header_set: null argument");
  std::string h (header, strnlen (header, header_cap));
  size_t key, tail;   // the line is rewritten from key, keeping h[tail:]
  bool append_newline = false;
  const char* found = header_find (h.c_str (), keyword);
  if (found)
  {
    key = size_t (found - h.c_str ());
    tail = key + strcspn (found, "#\n");
  }
  else
  {
    const size_t data = h.find ("DATA\n");
    key = tail = data != std::string::npos ? data : h.size ();
    append_newline = data == std::string::npos;
  }
  char line[8192];
  const int n = snprintf (line, sizeof (line), "%-12s %-20s   ", keyword, value);
  if (n < 0 || size_t (n) >= sizeof (line))
    return host_fail (DSPSR_B200_EINVAL, "ascii_header_set: value of %s too long", keyword);
  std::string out = h.substr (0, key) + line + (append_newline ? std::string ("\n") : h.substr (tail));
  if (out.size () + 1 > header_cap)
    return host_fail (DSPSR_B200_ETOOBIG, "ascii_header_set: %s needs %llu bytes, buffer has %llu",
                      keyword, (unsigned long long) out.size () + 1, (unsigned long long) header_cap);
  memcpy (header, out.c_str (), out.size () + 1);
  return DSPSR_B200_OK;
}

int dspsr_b200_dada_parse (const char* header, uint64_t header_bytes, dspsr_b200_dada_info* info)
{
  if (!header || !info)
    return host_fail (DSPSR_B200_EINVAL, "dada_parse: null argument");
  dspsr_b200_dada_info o;
  memset (&o, 0, sizeof (o));
  o.header_bytes = header_bytes;
  o.dual_sideband = -1;

  // ASCIIObservation::ascii_header_check (ASCIIObservation.h:134-143): a
  // required keyword that does not scan is an error
  auto required = [&] (const char* key, int rv) -> int {
    if (rv > 0) return DSPSR_B200_OK;
    return host_fail (DSPSR_B200_EINVAL, "ASCIIObservation: failed load %s", key);
  };
  std::string t;
  double d = 0;
  int64_t i = 0;
  int rc;

  // HDR_VERSION (:104-117) -- not required
  if (header_double (header, "HDR_VERSION", &d) == 1) o.hdr_version = d;

  // TELESCOPE, RECEIVER, SOURCE, MODE (:131-158)
  rc = header_token (header, "TELESCOPE", t);
  if ((rc = required ("TELESCOPE", rc))) return rc;
  copy_value (o.telescope, t);
  copy_value (o.receiver, header_token (header, "RECEIVER", t) > 0 ? t : std::string ("unknown"));
  rc = header_token (header, "SOURCE", t);
  if ((rc = required ("SOURCE", rc))) return rc;
  copy_value (o.source, t);
  if (header_token (header, "MODE", t) > 0) copy_value (o.mode, t);

  // FREQ, BW (:186-202)
  rc = header_double (header, "FREQ", &d);
  if ((rc = required ("FREQ", rc))) return rc;
  o.centre_freq_mhz = d;
  rc = header_double (header, "BW", &d);
  if ((rc = required ("BW", rc))) return rc;
  o.bandwidth_mhz = d;

  // NCHAN (default 1), NPOL, NBIT, NDIM (default 1) (:206-254)
  o.nchan = header_int64 (header, "NCHAN", &i) == 1 ? unsigned (i) : 1;
  rc = header_int64 (header, "NPOL", &i);
  if ((rc = required ("NPOL", rc))) return rc;
  o.npol = unsigned (i);
  rc = header_int64 (header, "NBIT", &i);
  if ((rc = required ("NBIT", rc))) return rc;
  o.nbit = unsigned (i);
  o.ndim = header_int64 (header, "NDIM", &i) == 1 ? unsigned (i) : 1;
  if (o.ndim != 1 && o.ndim != 2 && o.ndim != 4)
    return host_fail (DSPSR_B200_EINVAL, "ASCIIObservation: invalid NDIM=%u", o.ndim);

  // NDAT (:258-274), STATE, BASIS, DSB (:276-306)
  uint64_t u = 0;
  if (header_uint64 (header, "NDAT", &u) == 1) o.ndat = u;
  if (header_token (header, "STATE", t) > 0) copy_value (o.state, t);
  if (header_token (header, "BASIS", t) > 0) copy_value (o.basis, t);
  if (header_int64 (header, "DSB", &i) == 1) o.dual_sideband = i == 1 ? 1 : 0;

  // TSAMP in microseconds (:308-318)
  rc = header_double (header, "TSAMP", &d);
  if ((rc = required ("TSAMP", rc))) return rc;
  o.tsamp_us = d;
  o.rate_hz = 1.0 / (d * 1e-6);

  // UTC_START (:320-345): "TBD" leaves the start time unknown
  rc = header_token (header, "UTC_START", t);
  if ((rc = required ("UTC_START", rc))) return rc;
  copy_value (o.utc_start, t);
  bool have_start = false;
  if (t != "TBD")
  {
    if (!utc_to_mjd (t.c_str (), &o.start_day, &o.start_sec))
      return host_fail (DSPSR_B200_EINVAL, "ASCIIObservation: failed strptime (%s)", t.c_str ());
    have_start = true;
  }

  // BLOCK_DATA_BYTES: data interleaved with block headers (BlockSize.C:15-49)
  if (header_uint64 (header, "BLOCK_DATA_BYTES", &u) >= 0
      && (header_uint64 (header, "BLOCK_HEADER_BYTES", &u) == 1
          || header_uint64 (header, "BLOCK_TAILER_BYTES", &u) == 1))
    return host_fail (DSPSR_B200_EINVAL,
                      "dada_parse: block headers/tailers (BLOCK_DATA_BYTES) are not supported");

  // PICOSECONDS (:375-382), then OBS_OFFSET or OFFSET (:387-399)
  if (header_int64 (header, "PICOSECONDS", &i) == 1)
  {
    o.picoseconds = i;
    if (have_start) mjd_add (&o.start_day, &o.start_sec, &o.start_frac, double (i) / 1e12);
  }
  u = 0;
  if (header_uint64 (header, "OBS_OFFSET", &u) == 1)
    o.obs_offset = u;
  else if (header_uint64 (header, "OFFSET", &u) >= 0)
    o.obs_offset = u;
  else
    return host_fail (DSPSR_B200_EINVAL, "ASCIIObservation: failed load OBS_OFFSET");

  o.bits_per_sample = uint64_t (o.nbit) * o.npol * o.nchan * o.ndim;
  if (o.bits_per_sample == 0)
    return host_fail (DSPSR_B200_EINVAL, "dada_parse: zero bits per sample");

  // start time of sample 0 (:403-407): nsamples(offset_bytes) * sampling interval
  if (have_start)
  {
    const uint64_t offset_samples = (o.obs_offset * 8) / o.bits_per_sample;
    mjd_add (&o.start_day, &o.start_sec, &o.start_frac, double (offset_samples) * (d * 1e-6));
  }

  // INSTRUMENT (:413-416)
  if (header_token (header, "INSTRUMENT", t) > 0) copy_value (o.instrument, t);

  *info = o;
  return DSPSR_B200_OK;
}

int dspsr_b200_dada_open (const char* filename, dspsr_b200_dada_file** file,
                          dspsr_b200_dada_info* info)
{
  if (!filename || !file)
    return host_fail (DSPSR_B200_EINVAL, "dada_open: null argument");
  *file = nullptr;
  std::string header;
  uint64_t hdr_size = 0;
  int adjacent = 0;
  int rc = load_header (filename, header, &hdr_size, &adjacent);
  if (rc) return rc;
  if (header.empty () || header[0] == '\0')
    return host_fail (DSPSR_B200_EINVAL, "dada_open: empty header in %s", filename);

  dspsr_b200_dada_info o;
  rc = dspsr_b200_dada_parse (header.c_str (), hdr_size, &o);
  if (rc) return rc;
  o.adjacent_header = adjacent;

  const int fd = open (filename, O_RDONLY);
  if (fd < 0)
    return host_fail (DSPSR_B200_EINVAL, "open (%s): %s", filename, strerror (errno));
  struct stat st;
  if (fstat (fd, &st) != 0)
  {
    close (fd);
    return host_fail (DSPSR_B200_EINVAL, "fstat (%s): %s", filename, strerror (errno));
  }
  // File::fstat_file_ndat (File.C:366-390)
  if (uint64_t (st.st_size) < hdr_size)
  {
    close (fd);
    return host_fail (DSPSR_B200_EINVAL, "%s: file size=%lld < header size=%llu", filename,
                      (long long) st.st_size, (unsigned long long) hdr_size);
  }
  const uint64_t data_bytes = uint64_t (st.st_size) - hdr_size;
  o.file_ndat = data_bytes * 8 / o.bits_per_sample;
  // File::open (File.C:187-188): NDAT from the header, else from the file
  if (o.ndat == 0)
    o.ndat = o.file_ndat;

  dspsr_b200_dada_file* f = new dspsr_b200_dada_file;
  f->fd = fd;
  f->header = std::move (header);
  f->info = o;
  // File::load_bytes (File.C:261-272) stops at nbytes(ndat) + header_bytes;
  // a file shorter than NDAT says ends where the file does
  f->data_end = hdr_size + std::min<uint64_t> (o.ndat, o.file_ndat) * o.bits_per_sample / 8;
  *file = f;
  if (info) *info = o;
  return DSPSR_B200_OK;
}

int dspsr_b200_dada_is_valid (const char* filename)
{
  if (!filename) return 0;
  std::string header;
  uint64_t hdr_size = 0;
  int adjacent = 0;
  if (load_header (filename, header, &hdr_size, &adjacent)) return 0;
  if (header.empty () || header[0] == '\0') return 0;
  std::string t;
  double v;
  if (header_double (header.c_str (), "HDR_VERSION", &v) < 0) return 0;
  if (header_token (header.c_str (), "INSTRUMENT", t) < 0) return 0;
  return 1;
}

int dspsr_b200_dada_header (const dspsr_b200_dada_file* file, const char** text, uint64_t* size)
{
  if (!file || !text)
    return host_fail (DSPSR_B200_EINVAL, "dada_header: null argument");
  *text = file->header.c_str ();
  if (size) *size = file->header.size ();
  return DSPSR_B200_OK;
}

int dspsr_b200_dada_read (dspsr_b200_dada_file* file, uint64_t start_sample, uint64_t nsamp,
                          void* dst, uint64_t* nread)
{
  if (!file || (!dst && nsamp))
    return host_fail (DSPSR_B200_EINVAL, "dada_read: null argument");
  if (nread) *nread = 0;
  const uint64_t bits = file->info.bits_per_sample;
  if ((start_sample * bits) % 8 || (nsamp * bits) % 8)
    return host_fail (DSPSR_B200_EINVAL, "dada_read: %llu bits per sample do not end on a byte",
                      (unsigned long long) bits);
  const uint64_t begin = file->info.header_bytes + start_sample * bits / 8;
  if (begin >= file->data_end || nsamp == 0)
    return DSPSR_B200_OK;
  const uint64_t bytes = std::min<uint64_t> (nsamp * bits / 8, file->data_end - begin);
  // only whole samples are handed on
  const uint64_t want = bytes * 8 / bits * bits / 8;
  char* out = static_cast<char*> (dst);
  // Large reads are split over threads: one thread copying out of the page
  // cache moves ~6 GB/s, below the host link the blocks go to next.
  constexpr uint64_t CHUNK_MIN = 16ull << 20;
  const unsigned hw = std::max (1u, std::thread::hardware_concurrency ());
  const unsigned nthr = unsigned (std::min<uint64_t> ({16, hw, std::max<uint64_t> (1, want / CHUNK_MIN)}));
  const uint64_t per = (want / nthr + 4095) / 4096 * 4096;
  std::vector<uint64_t> got (nthr, 0);
  std::vector<int> err (nthr, 0);
  auto work = [&] (unsigned i) {
    const uint64_t lo = std::min<uint64_t> (want, i * per);
    const uint64_t hi = i + 1 == nthr ? want : std::min<uint64_t> (want, lo + per);
    uint64_t done = 0;
    while (lo + done < hi)
    {
      const ssize_t r = pread (file->fd, out + lo + done, size_t (hi - lo - done),
                               off_t (begin + lo + done));
      if (r < 0)
      {
        if (errno == EINTR) continue;
        err[i] = errno;
        break;
      }
      if (r == 0)
        break;
      done += uint64_t (r);
    }
    got[i] = done;
  };
  if (nthr == 1)
    work (0);
  else
  {
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < nthr; i++) pool.emplace_back (work, i);
    for (auto& t : pool) t.join ();
  }
  // the samples read: the prefix up to the first short chunk
  uint64_t done = 0;
  for (unsigned i = 0; i < nthr; i++)
  {
    if (err[i])
      return host_fail (DSPSR_B200_EINVAL, "dada_read: pread: %s", strerror (err[i]));
    done += got[i];
    const uint64_t lo = std::min<uint64_t> (want, i * per);
    const uint64_t hi = i + 1 == nthr ? want : std::min<uint64_t> (want, lo + per);
    if (got[i] < hi - lo) break;
  }
  if (nread) *nread = done * 8 / bits;
  return DSPSR_B200_OK;
}

int dspsr_b200_dada_close (dspsr_b200_dada_file* file)
{
  if (!file) return DSPSR_B200_EINVAL;
  if (file->fd >= 0) close (file->fd);
  delete file;
  return DSPSR_B200_OK;
}

}  // extern "C"

namespace dspsr_b200_host
{
const dspsr_b200_dada_info& dada_info (const dspsr_b200_dada_file* file)
{
  return file->info;
}
}  // namespace dspsr_b200_host
