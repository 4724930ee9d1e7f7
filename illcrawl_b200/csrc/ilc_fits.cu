// ilc_fits.cu -- FITS image output for rendered images and cubes (host code).
//
// illcrawl_render writes its results through util::fits (fits.hpp:215-258,
// cfitsio's fits_create_img + fits_write_pix, float images) and then appends
// its settings as header keys through util::fits_header::add_entry
// (fits.hpp:142-200: a COMMENT card with the entry's comment, then the key).
// This writer produces the same structure directly, without cfitsio: one
// primary HDU, BITPIX = -32, NAXIS1 = x (fastest), NAXIS2 = y, NAXIS3 = bins
// or frames, big-endian IEEE floats, header and data padded to 2880-byte
// records, keys longer than 8 characters (the reference's "integration.rel_tol"
// and the like) as ESO HIERARCH cards. It follows the FITS 4.0 standard; byte
// identity with cfitsio's output is not pinned (cfitsio is not available
// here, and the reference's header also records its OpenCL device).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ilc.h"

namespace {

std::string pad80(const std::string& s) {
  std::string r = s.substr(0, 80);
  r.resize(80, ' ');
  return r;
}

// "KEY     = " + value right-justified to column 30 (fixed format) + comment
std::string card(const std::string& key, const std::string& value, bool right_justify,
                 const std::string& comment) {
  std::string s;
  if (key.size() <= 8 && key.find_first_not_of("ABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789-_") ==
                             std::string::npos) {
    s = key;
    s.resize(8, ' ');
    s += "= ";
    if (right_justify && value.size() < 20) s += std::string(20 - value.size(), ' ');
    s += value;
  } else {
    s = "HIERARCH " + key + " = " + value;
  }
  if (!comment.empty() && s.size() + 3 < 80) s += " / " + comment;
  return pad80(s);
}

std::string quote(const std::string& v) {
  std::string r = "'";
  for (char ch : v) {
    r += ch;
    if (ch == '\'') r += '\'';
  }
  while (r.size() < 9) r += ' ';  // at least 8 characters between the quotes
  return r + "'";
}

std::string fmt_double(double v) {
  char buf[40];
  std::snprintf(buf, sizeof buf, "%.15G", v);
  std::string s = buf;
  if (s.find_first_of(".EN") == std::string::npos) s += ".";
  return s;
}

}  // namespace

extern "C" ilc_status ilc_fits_write_image(const char* path, const float* data, int32_t naxis,
                                           const int64_t* naxes, const ilc_fits_card* cards,
                                           int32_t n_cards) {
  if (!path || !data || naxis < 1 || naxis > 3 || !naxes || n_cards < 0 ||
      (n_cards > 0 && !cards))
    return ILC_ERR_INVALID_ARGUMENT;
  uint64_t count = 1;
  for (int i = 0; i < naxis; ++i) {
    if (naxes[i] < 1) return ILC_ERR_INVALID_ARGUMENT;
    count *= (uint64_t)naxes[i];
  }
  std::vector<std::string> h;
  h.push_back(card("SIMPLE", "T", true, "file does conform to FITS standard"));
  h.push_back(card("BITPIX", "-32", true, "number of bits per data pixel"));
  h.push_back(card("NAXIS", std::to_string(naxis), true, "number of data axes"));
  for (int i = 0; i < naxis; ++i)
    h.push_back(card("NAXIS" + std::to_string(i + 1), std::to_string(naxes[i]), true,
                     "length of data axis " + std::to_string(i + 1)));
  h.push_back(card("EXTEND", "T", true, "FITS dataset may contain extensions"));
  for (int32_t k = 0; k < n_cards; ++k) {
    const ilc_fits_card& c = cards[k];
    if (!c.key || !*c.key) return ILC_ERR_INVALID_ARGUMENT;
    if (c.comment && *c.comment) h.push_back(pad80(std::string("COMMENT ") + c.comment));
    std::string v;
    bool right = true;
    switch (c.type) {
      case ILC_FITS_DOUBLE: v = fmt_double(c.number); break;
      case ILC_FITS_INTEGER: v = std::to_string(c.integer); break;
      case ILC_FITS_LOGICAL: v = c.integer ? "T" : "F"; break;
      case ILC_FITS_STRING:
        v = quote(c.text ? c.text : "");
        right = false;
        break;
      default: return ILC_ERR_INVALID_ARGUMENT;
    }
    h.push_back(card(c.key, v, right, ""));
  }
  h.push_back(pad80("END"));
  std::string head;
  for (const auto& s : h) head += s;
  head.resize(((head.size() + 2879) / 2880) * 2880, ' ');
  FILE* f = std::fopen(path, "wb");
  if (!f) return ILC_ERR_INVALID_ARGUMENT;
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  std::vector<unsigned char> buf(1 << 16);
  uint64_t done = 0;
  while (ok && done < count) {
    const uint64_t m = std::min<uint64_t>(count - done, buf.size() / 4);
    for (uint64_t i = 0; i < m; ++i) {
      uint32_t u;
      std::memcpy(&u, &data[done + i], 4);
      buf[4 * i] = (unsigned char)(u >> 24);
      buf[4 * i + 1] = (unsigned char)(u >> 16);
      buf[4 * i + 2] = (unsigned char)(u >> 8);
      buf[4 * i + 3] = (unsigned char)u;
    }
    ok = std::fwrite(buf.data(), 1, 4 * m, f) == 4 * m;
    done += m;
  }
  const uint64_t tail = (2880 - (count * 4) % 2880) % 2880;
  if (ok && tail) {
    std::vector<unsigned char> z(tail, 0);
    ok = std::fwrite(z.data(), 1, tail, f) == tail;
  }
  if (std::fclose(f) != 0) ok = false;
  return ok ? ILC_OK : ILC_ERR_INTERNAL;
}
