// Minimal FITS image I/O: 2880-byte records, 80-character header cards,
// big-endian data; BITPIX 8/16/32/64/-32/-64 read with BSCALE/BZERO.
#include "fits_io.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace {

constexpr size_t kBlock = 2880;
constexpr size_t kCard = 80;

std::string card_key(const char* c) {
  std::string k(c, 8);
  while (!k.empty() && k.back() == ' ') k.pop_back();
  return k;
}

std::string card_value(const char* c) {
  if (std::strncmp(c + 8, "= ", 2) != 0) return "";
  std::string v(c + 10, kCard - 10);
  size_t p = 0;
  while (p < v.size() && v[p] == ' ') ++p;
  if (p < v.size() && v[p] == '\'') {
    size_t q = v.find('\'', p + 1);
    std::string s = v.substr(p + 1, q == std::string::npos ? std::string::npos : q - p - 1);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    return s;
  }
  size_t slash = v.find('/', p);
  std::string s = v.substr(p, slash == std::string::npos ? std::string::npos : slash - p);
  while (!s.empty() && s.back() == ' ') s.pop_back();
  return s;
}

template <typename T>
T be_load(const unsigned char* p) {
  unsigned char b[sizeof(T)];
  for (size_t i = 0; i < sizeof(T); ++i) b[i] = p[sizeof(T) - 1 - i];
  T v;
  std::memcpy(&v, b, sizeof(T));
  return v;
}

// A string-valued card: the quoted value starts in column 11, padded to at
// least 8 characters inside the quotes.
void put_str_card(std::string& h, const std::string& key, const std::string& value) {
  std::string v = value;
  if (v.size() < 8) v.resize(8, ' ');
  std::string c = key;
  c.resize(8, ' ');
  c += "= '" + v + "'";
  c.resize(kCard, ' ');
  h += c;
}

void be_store32(unsigned char* d, const void* src) {
  unsigned char b[4];
  std::memcpy(b, src, 4);
  d[0] = b[3];
  d[1] = b[2];
  d[2] = b[1];
  d[3] = b[0];
}

void put_card(std::string& h, const std::string& key, const std::string& value) {
  char buf[kCard + 1];
  if (value.empty())
    std::snprintf(buf, sizeof(buf), "%-8.8s", key.c_str());
  else
    std::snprintf(buf, sizeof(buf), "%-8.8s= %20s", key.c_str(), value.c_str());
  std::string c(buf);
  c.resize(kCard, ' ');
  h += c;
}

}  // namespace

bool fits_read_all(const std::string& path, std::vector<FitsImage>& hdus, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::vector<unsigned char> buf((std::istreambuf_iterator<char>(f)),
                                 std::istreambuf_iterator<char>());
  size_t pos = 0;
  hdus.clear();
  while (pos + kBlock <= buf.size()) {
    int bitpix = 0, naxis = 0;
    std::vector<long> naxes;
    double bscale = 1.0, bzero = 0.0;
    long pcount = 0, gcount = 1;
    std::string extname, xtension;
    bool end = false;
    size_t hpos = pos;
    while (!end) {
      if (hpos + kBlock > buf.size()) {
        err = "truncated FITS header in " + path;
        return false;
      }
      for (size_t c = 0; c < kBlock / kCard; ++c) {
        const char* card = reinterpret_cast<const char*>(&buf[hpos + c * kCard]);
        std::string key = card_key(card);
        if (key == "END") {
          end = true;
          break;
        }
        std::string val = card_value(card);
        if (key == "BITPIX") bitpix = std::atoi(val.c_str());
        else if (key == "NAXIS") naxis = std::atoi(val.c_str());
        else if (key.rfind("NAXIS", 0) == 0 && key.size() > 5) {
          int ax = std::atoi(key.c_str() + 5);
          if (ax >= 1) {
            if ((int)naxes.size() < ax) naxes.resize(ax, 0);
            naxes[ax - 1] = std::atol(val.c_str());
          }
        } else if (key == "BSCALE") bscale = std::atof(val.c_str());
        else if (key == "BZERO") bzero = std::atof(val.c_str());
        else if (key == "PCOUNT") pcount = std::atol(val.c_str());
        else if (key == "GCOUNT") gcount = std::atol(val.c_str());
        else if (key == "EXTNAME") extname = val;
        else if (key == "XTENSION") xtension = val;
      }
      hpos += kBlock;
    }
    naxes.resize(naxis > 0 ? naxis : 0);
    size_t count = naxis > 0 ? 1 : 0;
    for (long a : naxes) count *= (size_t)a;
    const size_t bpe = (size_t)(bitpix < 0 ? -bitpix : bitpix) / 8;
    const size_t nbytes = bpe * gcount * (pcount + count);
    FitsImage img;
    img.naxes = naxes;
    img.extname = extname;
    if (xtension.empty() || xtension == "IMAGE") {
      if (hpos + count * bpe > buf.size()) {
        err = "truncated FITS data in " + path;
        return false;
      }
      img.data.resize(count);
      const unsigned char* d = &buf[hpos];
      for (size_t i = 0; i < count; ++i) {
        double v;
        switch (bitpix) {
          case 8: v = d[i]; break;
          case 16: v = be_load<int16_t>(d + 2 * i); break;
          case 32: v = be_load<int32_t>(d + 4 * i); break;
          case 64: v = (double)be_load<int64_t>(d + 8 * i); break;
          case -32: v = be_load<float>(d + 4 * i); break;
          case -64: v = be_load<double>(d + 8 * i); break;
          default:
            err = "unsupported BITPIX " + std::to_string(bitpix) + " in " + path;
            return false;
        }
        img.data[i] = (float)(bzero + bscale * v);
      }
    }
    hdus.push_back(std::move(img));
    pos = hpos + ((nbytes + kBlock - 1) / kBlock) * kBlock;
  }
  if (hdus.empty()) {
    err = "no FITS HDU in " + path;
    return false;
  }
  return true;
}

bool fits_read_image(const std::string& path, FitsImage& img, std::string& err) {
  std::vector<FitsImage> hdus;
  if (!fits_read_all(path, hdus, err)) return false;
  for (auto& h : hdus) {
    if (h.data.empty()) continue;
    if (h.naxes.size() != 1 && h.naxes.size() != 2) {
      err = "unsupported NAXIS=" + std::to_string(h.naxes.size()) + " for file " + path;
      return false;
    }
    img = std::move(h);
    if (img.naxes.size() == 1) img.naxes.push_back(1);
    return true;
  }
  err = "no image data in " + path;
  return false;
}

bool fits_write_image(const std::string& path, const float* data, const std::vector<long>& naxes,
                      std::string& err) {
  std::string h;
  put_card(h, "SIMPLE", "T");
  put_card(h, "BITPIX", "-32");
  put_card(h, "NAXIS", std::to_string(naxes.size()));
  size_t count = 1;
  for (size_t a = 0; a < naxes.size(); ++a) {
    put_card(h, "NAXIS" + std::to_string(a + 1), std::to_string(naxes[a]));
    count *= (size_t)naxes[a];
  }
  put_card(h, "END", "");
  h.resize(((h.size() + kBlock - 1) / kBlock) * kBlock, ' ');
  std::vector<unsigned char> d(((count * 4 + kBlock - 1) / kBlock) * kBlock, 0);
  for (size_t i = 0; i < count; ++i) {
    unsigned char b[4];
    std::memcpy(b, &data[i], 4);
    d[4 * i + 0] = b[3];
    d[4 * i + 1] = b[2];
    d[4 * i + 2] = b[1];
    d[4 * i + 3] = b[0];
  }
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) {
    err = "cannot create " + path;
    return false;
  }
  f.write(h.data(), (std::streamsize)h.size());
  f.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)d.size());
  if (!f) {
    err = "write failed for " + path;
    return false;
  }
  return true;
}

bool fits_write_table(const std::string& path, const std::vector<FitsColumn>& cols, size_t nrows,
                      const std::string& extname, std::string& err) {
  for (const FitsColumn& c : cols)
    if (c.form != 'J' && c.form != 'E') {
      err = "unsupported column form for " + c.name;
      return false;
    }
  std::string h;
  put_card(h, "SIMPLE", "T");
  put_card(h, "BITPIX", "8");
  put_card(h, "NAXIS", "0");
  put_card(h, "EXTEND", "T");
  put_card(h, "END", "");
  h.resize(((h.size() + kBlock - 1) / kBlock) * kBlock, ' ');
  const size_t row_bytes = 4 * cols.size();
  std::string x;
  put_str_card(x, "XTENSION", "BINTABLE");
  put_card(x, "BITPIX", "8");
  put_card(x, "NAXIS", "2");
  put_card(x, "NAXIS1", std::to_string(row_bytes));
  put_card(x, "NAXIS2", std::to_string(nrows));
  put_card(x, "PCOUNT", "0");
  put_card(x, "GCOUNT", "1");
  put_card(x, "TFIELDS", std::to_string(cols.size()));
  for (size_t k = 0; k < cols.size(); ++k) {
    put_str_card(x, "TTYPE" + std::to_string(k + 1), cols[k].name);
    put_str_card(x, "TFORM" + std::to_string(k + 1), std::string("1") + cols[k].form);
  }
  put_str_card(x, "EXTNAME", extname);
  put_card(x, "END", "");
  x.resize(((x.size() + kBlock - 1) / kBlock) * kBlock, ' ');
  std::vector<unsigned char> d(((row_bytes * nrows + kBlock - 1) / kBlock) * kBlock, 0);
  for (size_t r = 0; r < nrows; ++r)
    for (size_t k = 0; k < cols.size(); ++k)
      be_store32(&d[r * row_bytes + 4 * k], static_cast<const char*>(cols[k].data) + 4 * r);
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) {
    err = "cannot create " + path;
    return false;
  }
  f.write(h.data(), (std::streamsize)h.size());
  f.write(x.data(), (std::streamsize)x.size());
  f.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)d.size());
  if (!f) {
    err = "write failed for " + path;
    return false;
  }
  return true;
}

bool fits_read_combined(const std::string& path, CombinedInput& in, std::string& err) {
  std::vector<FitsImage> hdus;
  if (!fits_read_all(path, hdus, err)) return false;
  const FitsImage *tm = nullptr, *vis = nullptr, *rc = nullptr;
  for (const FitsImage& h : hdus) {
    if (h.extname == "TRANSFORMATION MATRICES") tm = &h;
    else if (h.extname == "VISIBILITIES") vis = &h;
    else if (h.extname == "R-COORDINATES") rc = &h;
  }
  if (!tm || !vis || !rc) {
    err = path + " lacks one of the extensions TRANSFORMATION MATRICES, VISIBILITIES, "
                 "R-COORDINATES";
    return false;
  }
  if (tm->naxes.size() != 3 || tm->naxes[0] != 3 || tm->naxes[1] != 3 ||
      vis->naxes.size() != 3 || vis->naxes[0] != 2 || rc->naxes != vis->naxes ||
      vis->naxes[2] != tm->naxes[2]) {
    err = "unexpected extension shapes in " + path;
    return false;
  }
  in.snapshots = (size_t)tm->naxes[2];
  in.samples = (size_t)vis->naxes[1];
  const size_t ns = in.snapshots * in.samples;
  in.V = tm->data;
  in.B = rc->data;
  in.vis_re.resize(ns);
  in.vis_im.resize(ns);
  for (size_t k = 0; k < ns; ++k) {
    in.vis_re[k] = vis->data[2 * k];
    in.vis_im[k] = vis->data[2 * k + 1];
  }
  return true;
}
