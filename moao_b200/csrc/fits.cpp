// Minimal FITS image I/O (primary HDU, 1-D or 2-D images), for the inputs the
// reference reads with cfitsio (Dx, idx, abs2fi, otftel: common/io/fits.cpp,
// common/tomo_struct/intersample.cpp:208-300) and the matrices its check
// program writes. FITS standard 4.0: 2880-byte blocks of 80-character header
// cards, big-endian data, NAXIS1 the fastest-varying axis, physical value =
// BZERO + BSCALE * stored value.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "moao_internal.h"

namespace moao {
namespace {

constexpr size_t kBlock = 2880;
constexpr size_t kCard = 80;

struct Header {
  int bitpix = 0;
  int naxis = 0;
  long naxes[2] = {1, 1};
  double bzero = 0, bscale = 1;
  size_t data_offset = 0;
};

std::string card_key(const char* c) {
  std::string k(c, 8);
  while (!k.empty() && k.back() == ' ') k.pop_back();
  return k;
}

// Value field of a card (after "= "), comment stripped.
std::string card_value(const char* c) {
  std::string v(c + 10, kCard - 10);
  const size_t slash = v.find('/');
  if (slash != std::string::npos) v = v.substr(0, slash);
  const size_t a = v.find_first_not_of(' '), b = v.find_last_not_of(' ');
  return a == std::string::npos ? std::string() : v.substr(a, b - a + 1);
}

moao_status read_header(FILE* f, const char* path, Header* h) {
  std::vector<char> blk(kBlock);
  bool simple = false, end = false;
  size_t blocks = 0;
  while (!end) {
    if (fread(blk.data(), 1, kBlock, f) != kBlock)
      return set_error(MOAO_ERR_IO, std::string("fits: truncated header in ") + path);
    ++blocks;
    for (size_t c = 0; c < kBlock / kCard && !end; ++c) {
      const char* card = blk.data() + c * kCard;
      const std::string key = card_key(card);
      if (blocks == 1 && c == 0) {
        simple = key == "SIMPLE" && card_value(card) == "T";
        if (!simple) return set_error(MOAO_ERR_IO, std::string("fits: not a FITS file: ") + path);
        continue;
      }
      if (key == "END") {
        end = true;
      } else if (key == "BITPIX") {
        h->bitpix = std::stoi(card_value(card));
      } else if (key == "NAXIS") {
        h->naxis = std::stoi(card_value(card));
      } else if (key == "NAXIS1") {
        h->naxes[0] = std::stol(card_value(card));
      } else if (key == "NAXIS2") {
        h->naxes[1] = std::stol(card_value(card));
      } else if (key == "BZERO") {
        h->bzero = std::stod(card_value(card));
      } else if (key == "BSCALE") {
        h->bscale = std::stod(card_value(card));
      }
    }
  }
  if (h->naxis < 1 || h->naxis > 2)
    return set_error(MOAO_ERR_UNSUPPORTED, std::string("fits: only 1-D and 2-D images: ") + path);
  const int b = h->bitpix;
  if (b != 8 && b != 16 && b != 32 && b != 64 && b != -32 && b != -64)
    return set_error(MOAO_ERR_IO, std::string("fits: bad BITPIX in ") + path);
  if (h->naxis == 1) h->naxes[1] = 1;
  h->data_offset = blocks * kBlock;
  return MOAO_OK;
}

template <typename V>
V from_big_endian(const unsigned char* p) {
  unsigned char b[sizeof(V)];
  for (size_t i = 0; i < sizeof(V); ++i) b[i] = p[sizeof(V) - 1 - i];
  V v;
  std::memcpy(&v, b, sizeof(V));
  return v;
}

template <typename V>
void to_big_endian(V v, unsigned char* p) {
  unsigned char b[sizeof(V)];
  std::memcpy(b, &v, sizeof(V));
  for (size_t i = 0; i < sizeof(V); ++i) p[i] = b[sizeof(V) - 1 - i];
}

// Reads the image converted to Out (integer BITPIX without scaling stays exact
// for Out = long long).
template <typename Out>
moao_status read_image(const char* path, long* n1, long* n2, Out* out, long cap) {
  if (!path || !n1 || !n2) return set_error(MOAO_ERR_BAD_ARG, "fits_read: null argument");
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MOAO_ERR_IO, std::string("fits: cannot open ") + path);
  Header h;
  moao_status st = read_header(f, path, &h);
  if (st != MOAO_OK) {
    fclose(f);
    return st;
  }
  *n1 = h.naxes[0];
  *n2 = h.naxes[1];
  const size_t count = (size_t)h.naxes[0] * (size_t)h.naxes[1];
  if (!out) {
    fclose(f);
    return MOAO_OK;
  }
  if ((long)count > cap) {
    fclose(f);
    return set_error(MOAO_ERR_BAD_ARG, std::string("fits: buffer too small for ") + path);
  }
  const size_t es = (size_t)std::abs(h.bitpix) / 8;
  std::vector<unsigned char> raw(count * es);
  if (fseek(f, (long)h.data_offset, SEEK_SET) != 0 || fread(raw.data(), 1, raw.size(), f) != raw.size()) {
    fclose(f);
    return set_error(MOAO_ERR_IO, std::string("fits: truncated data in ") + path);
  }
  fclose(f);
  const bool scaled = h.bzero != 0 || h.bscale != 1;
  for (size_t i = 0; i < count; ++i) {
    const unsigned char* p = raw.data() + i * es;
    switch (h.bitpix) {
      case 8: {
        const double v = (double)p[0];
        out[i] = (Out)(scaled ? h.bzero + h.bscale * v : v);
        break;
      }
      case 16: {
        const int16_t v = from_big_endian<int16_t>(p);
        out[i] = scaled ? (Out)(h.bzero + h.bscale * v) : (Out)v;
        break;
      }
      case 32: {
        const int32_t v = from_big_endian<int32_t>(p);
        out[i] = scaled ? (Out)(h.bzero + h.bscale * v) : (Out)v;
        break;
      }
      case 64: {
        const int64_t v = from_big_endian<int64_t>(p);
        out[i] = scaled ? (Out)(h.bzero + h.bscale * (double)v) : (Out)v;
        break;
      }
      case -32: {
        const float v = from_big_endian<float>(p);
        out[i] = (Out)(scaled ? h.bzero + h.bscale * v : v);
        break;
      }
      default: {
        const double v = from_big_endian<double>(p);
        out[i] = (Out)(scaled ? h.bzero + h.bscale * v : v);
        break;
      }
    }
  }
  return MOAO_OK;
}

void put_card(std::vector<char>& hdr, const std::string& text) {
  std::string c = text;
  c.resize(kCard, ' ');
  hdr.insert(hdr.end(), c.begin(), c.end());
}

std::string value_card(const char* key, const std::string& value, const char* comment) {
  char buf[kCard + 1];
  snprintf(buf, sizeof(buf), "%-8s= %20s / %s", key, value.c_str(), comment);
  return buf;
}

template <typename V>
moao_status write_image(const char* path, long n1, long n2, const V* data, int bitpix) {
  if (!path || !data || n1 <= 0 || n2 <= 0)
    return set_error(MOAO_ERR_BAD_ARG, "fits_write: bad arguments");
  std::vector<char> hdr;
  put_card(hdr, value_card("SIMPLE", "T", "file conforms to FITS standard"));
  put_card(hdr, value_card("BITPIX", std::to_string(bitpix), "bits per data value"));
  put_card(hdr, value_card("NAXIS", "2", "number of axes"));
  put_card(hdr, value_card("NAXIS1", std::to_string(n1), "fastest-varying axis"));
  put_card(hdr, value_card("NAXIS2", std::to_string(n2), "second axis"));
  put_card(hdr, "END");
  hdr.resize((hdr.size() + kBlock - 1) / kBlock * kBlock, ' ');
  const size_t count = (size_t)n1 * (size_t)n2;
  std::vector<unsigned char> raw(((count * sizeof(V)) + kBlock - 1) / kBlock * kBlock, 0);
  for (size_t i = 0; i < count; ++i) to_big_endian<V>(data[i], raw.data() + i * sizeof(V));
  FILE* f = fopen(path, "wb");
  if (!f) return set_error(MOAO_ERR_IO, std::string("fits: cannot create ") + path);
  const bool ok = fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() &&
                  fwrite(raw.data(), 1, raw.size(), f) == raw.size();
  const bool closed = fclose(f) == 0;
  if (!ok || !closed) return set_error(MOAO_ERR_IO, std::string("fits: write failed: ") + path);
  return MOAO_OK;
}

}  // namespace
}  // namespace moao

using namespace moao;

extern "C" {

moao_status moao_fits_read_f64(const char* path, long* naxis1, long* naxis2, double* out,
                               long cap) {
  return read_image<double>(path, naxis1, naxis2, out, cap);
}

moao_status moao_fits_read_i64(const char* path, long* naxis1, long* naxis2, long long* out,
                               long cap) {
  return read_image<long long>(path, naxis1, naxis2, out, cap);
}

moao_status moao_fits_write_f64(const char* path, long naxis1, long naxis2, const double* data) {
  return write_image<double>(path, naxis1, naxis2, data, -64);
}

moao_status moao_fits_write_i64(const char* path, long naxis1, long naxis2,
                                const long long* data) {
  return write_image<long long>(path, naxis1, naxis2, data, 64);
}

}  // extern "C"
