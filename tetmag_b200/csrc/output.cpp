// Output and restart artefacts of a tetmag run, host C++:
//
//  * write_vtu: the unstructured-grid file of MeshWriter::outputVTK (io/MeshWriter.cpp:174-239):
//    tetrahedra, point vectors "Magnetization", point scalars "Material", optionally a second point
//    vector field ("Demag" in TheSimulation.cpp:321), and the time as a one-value field array
//    ("timeInPs", io/MeshWriter.h:60).  Written as VTK XML, ASCII or appended raw binary, so that
//    VTK / ParaView and tetmag's own reader open it.
//  * read_magnetization: VTKReader::readMag / readMagGeneric / getTime (io/VTKReader.cpp:83-181):
//    the point array "Magnetization" and the field value "timeInPs" of a .vtu file (ASCII, inline
//    base64 or appended raw / base64 data, uncompressed or zlib-compressed, UInt32 or UInt64
//    headers, as VTK's XML writer produces) or of a legacy ASCII .vtk file.  The point count must
//    match (VTKReader::checkNodeNumber, :72-81).
//  * log_header / log_row: the columns of tetmag's .log file (writeLogFileHeader,
//    main/TheSimulation.cpp:85-93; TheSimulation::writeLogStream, :367-372), character for
//    character: iostream fixed / scientific / default-float formatting, and the vectors printed the
//    way Eigen prints a row vector (every coefficient right-aligned to the widest one, separated by
//    one space).
#include <zlib.h>

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "tmb.h"
#include "tmb_host.h"

namespace tmb {

namespace {

void put_f64(std::ostream& o, double v) {
  char b[32];
  std::snprintf(b, sizeof b, "%.17g", v);
  o << b;
}

struct Appended {
  std::string blob;   // UInt64 byte count + bytes, per array
  size_t add(const void* p, size_t nbytes) {
    const size_t off = blob.size();
    const uint64_t n = nbytes;
    blob.append(reinterpret_cast<const char*>(&n), sizeof n);
    blob.append(reinterpret_cast<const char*>(p), nbytes);
    return off;
  }
};

}  // namespace

int write_vtu(const std::string& path, int nx, const double* xyz, int ntet, const int* tets, const double* m,
              const int* material, double time_ps, const char* time_name, const double* field,
              const char* field_name, int binary, std::string& err) {
  std::ofstream f(path, std::ios::binary);
  if (!f) {
    err = "write_vtu: cannot open " + path;
    return TMB_ERR_ARG;
  }
  const std::string tname = time_name && *time_name ? time_name : "timeInPs";
  const std::string fname = field_name && *field_name ? field_name : "Demag";
  // row-major copies of the SoA vectors, the grid's connectivity as VTK wants it
  std::vector<double> mr(size_t(3) * nx), fr(field ? size_t(3) * nx : 0);
  for (int i = 0; i < nx; ++i)
    for (int d = 0; d < 3; ++d) {
      mr[size_t(3) * i + d] = m[size_t(d) * nx + i];
      if (field) fr[size_t(3) * i + d] = field[size_t(d) * nx + i];
    }
  std::vector<int32_t> mat(nx, 0);
  if (material)
    for (int i = 0; i < nx; ++i) mat[i] = material[i];
  std::vector<int64_t> conn(size_t(4) * ntet), offs(ntet);
  std::vector<uint8_t> types(ntet, 10);   // VTK_TETRA
  for (size_t k = 0; k < conn.size(); ++k) conn[k] = tets[k];
  for (int e = 0; e < ntet; ++e) offs[e] = int64_t(4) * (e + 1);

  Appended ap;
  auto array = [&](const char* type, const std::string& name, int ncomp, const void* data, size_t count,
                   size_t elem, auto&& ascii) {
    f << "        <DataArray type=\"" << type << "\" Name=\"" << name << "\"";
    if (ncomp > 1) f << " NumberOfComponents=\"" << ncomp << "\"";
    if (binary) {
      f << " format=\"appended\" offset=\"" << ap.add(data, count * elem) << "\"/>\n";
    } else {
      f << " format=\"ascii\">\n";
      for (size_t k = 0; k < count; ++k) {
        ascii(k);
        f << ((k + 1) % 12 == 0 || k + 1 == count ? "\n" : " ");
      }
      f << "        </DataArray>\n";
    }
  };
  f << "<?xml version=\"1.0\"?>\n";
  f << "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
  f << "  <UnstructuredGrid>\n    <FieldData>\n";
  f << "      <DataArray type=\"Float64\" Name=\"" << tname << "\" NumberOfTuples=\"1\" format=\"ascii\">\n        ";
  put_f64(f, time_ps);
  f << "\n      </DataArray>\n    </FieldData>\n";
  f << "    <Piece NumberOfPoints=\"" << nx << "\" NumberOfCells=\"" << ntet << "\">\n";
  f << "      <PointData Scalars=\"Material\" Vectors=\"Magnetization\">\n";
  array("Float64", "Magnetization", 3, mr.data(), mr.size(), 8, [&](size_t k) { put_f64(f, mr[k]); });
  array("Int32", "Material", 1, mat.data(), mat.size(), 4, [&](size_t k) { f << mat[k]; });
  if (field) array("Float64", fname, 3, fr.data(), fr.size(), 8, [&](size_t k) { put_f64(f, fr[k]); });
  f << "      </PointData>\n      <Points>\n";
  array("Float64", "Points", 3, xyz, size_t(3) * nx, 8, [&](size_t k) { put_f64(f, xyz[k]); });
  f << "      </Points>\n      <Cells>\n";
  array("Int64", "connectivity", 1, conn.data(), conn.size(), 8, [&](size_t k) { f << conn[k]; });
  array("Int64", "offsets", 1, offs.data(), offs.size(), 8, [&](size_t k) { f << offs[k]; });
  array("UInt8", "types", 1, types.data(), types.size(), 1, [&](size_t k) { f << int(types[k]); });
  f << "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n";
  if (binary) {
    f << "  <AppendedData encoding=\"raw\">\n   _";
    f.write(ap.blob.data(), std::streamsize(ap.blob.size()));
    f << "\n  </AppendedData>\n";
  }
  f << "</VTKFile>\n";
  if (!f) {
    err = "write_vtu: write failed on " + path;
    return TMB_ERR_ARG;
  }
  return TMB_OK;
}

// --------------------------------------------------------------------------------------------
// Reading
// --------------------------------------------------------------------------------------------
namespace {

struct ReadError {
  std::string msg;
};

[[noreturn]] void bad(const std::string& m) { throw ReadError{m}; }

std::string attr(const std::string& tag, const char* name) {
  const std::string key = std::string(name) + "=\"";
  size_t p = 0;
  while ((p = tag.find(key, p)) != std::string::npos) {
    if (p == 0 || std::isspace(static_cast<unsigned char>(tag[p - 1]))) {
      const size_t b = p + key.size(), e = tag.find('"', b);
      if (e == std::string::npos) bad("unterminated attribute " + std::string(name));
      return tag.substr(b, e - b);
    }
    p += key.size();
  }
  return "";
}

int type_size(const std::string& t) {
  if (t == "Float64" || t == "Int64" || t == "UInt64") return 8;
  if (t == "Float32" || t == "Int32" || t == "UInt32") return 4;
  if (t == "Int16" || t == "UInt16") return 2;
  if (t == "Int8" || t == "UInt8") return 1;
  bad("unsupported data type " + t);
}

double as_double(const std::string& t, const unsigned char* p) {
  if (t == "Float64") { double v; std::memcpy(&v, p, 8); return v; }
  if (t == "Float32") { float v; std::memcpy(&v, p, 4); return v; }
  if (t == "Int64") { int64_t v; std::memcpy(&v, p, 8); return double(v); }
  if (t == "UInt64") { uint64_t v; std::memcpy(&v, p, 8); return double(v); }
  if (t == "Int32") { int32_t v; std::memcpy(&v, p, 4); return v; }
  if (t == "UInt32") { uint32_t v; std::memcpy(&v, p, 4); return v; }
  if (t == "Int16") { int16_t v; std::memcpy(&v, p, 2); return v; }
  if (t == "UInt16") { uint16_t v; std::memcpy(&v, p, 2); return v; }
  if (t == "Int8") return double(*reinterpret_cast<const int8_t*>(p));
  return double(*p);
}

int b64_val(char c) {
  if (c >= 'A' && c <= 'Z') return c - 'A';
  if (c >= 'a' && c <= 'z') return c - 'a' + 26;
  if (c >= '0' && c <= '9') return c - '0' + 52;
  if (c == '+') return 62;
  if (c == '/') return 63;
  return -1;
}

// Base64 text without whitespace.
std::string b64_clean(const char* p, size_t n) {
  std::string s;
  s.reserve(n);
  for (size_t i = 0; i < n; ++i)
    if (!std::isspace(static_cast<unsigned char>(p[i]))) s.push_back(p[i]);
  return s;
}

// Decodes the base64 characters s[pos, pos + nchars) (nchars a multiple of 4).
std::vector<unsigned char> b64_decode(const std::string& s, size_t pos, size_t nchars) {
  if (pos + nchars > s.size() || nchars % 4) bad("truncated base64 data");
  std::vector<unsigned char> out;
  out.reserve(nchars / 4 * 3);
  for (size_t i = pos; i < pos + nchars; i += 4) {
    int v[4];
    int pad = 0;
    for (int k = 0; k < 4; ++k) {
      const char c = s[i + k];
      if (c == '=') {
        v[k] = 0;
        ++pad;
      } else if ((v[k] = b64_val(c)) < 0) {
        bad("invalid base64 character");
      }
    }
    const uint32_t w = (uint32_t(v[0]) << 18) | (uint32_t(v[1]) << 12) | (uint32_t(v[2]) << 6) | uint32_t(v[3]);
    out.push_back(static_cast<unsigned char>(w >> 16));
    if (pad < 2) out.push_back(static_cast<unsigned char>(w >> 8));
    if (pad < 1) out.push_back(static_cast<unsigned char>(w));
  }
  return out;
}

size_t b64_len(size_t nbytes) { return (nbytes + 2) / 3 * 4; }

uint64_t read_uint(const unsigned char* p, int hsize) {
  if (hsize == 8) {
    uint64_t v;
    std::memcpy(&v, p, 8);
    return v;
  }
  uint32_t v;
  std::memcpy(&v, p, 4);
  return v;
}

std::vector<unsigned char> inflate_blocks(const std::vector<uint64_t>& hdr, const unsigned char* data,
                                          size_t avail) {
  // hdr = {nblocks, block size, last block size, compressed size of each block}
  const uint64_t nb = hdr[0], bs = hdr[1], last = hdr[2];
  std::vector<unsigned char> out;
  size_t off = 0;
  for (uint64_t b = 0; b < nb; ++b) {
    const uint64_t csz = hdr[3 + b];
    const uint64_t usz = (b + 1 == nb && last != 0) ? last : bs;
    if (off + csz > avail) bad("truncated compressed block");
    const size_t o = out.size();
    out.resize(o + usz);
    uLongf dl = uLongf(usz);
    if (uncompress(out.data() + o, &dl, data + off, uLong(csz)) != Z_OK || dl != usz)
      bad("zlib block does not inflate to its stated size");
    off += csz;
  }
  return out;
}

struct XmlFile {
  std::string text;
  int hsize = 4;          // header_type UInt32 (VTK's default when the attribute is absent) or UInt64
  bool zlib = false;
  std::string app_enc;    // appended data encoding ("raw" / "base64"), empty if none
  size_t app_pos = 0;     // first byte after the '_' marker
};

// Payload bytes of a binary DataArray: inline base64 (text = element body) or appended at offset.
std::vector<unsigned char> binary_payload(const XmlFile& X, bool appended, const std::string& body, size_t offset) {
  const int hs = X.hsize;
  if (appended && X.app_enc == "raw") {
    const size_t p0 = X.app_pos + offset;
    const auto* base = reinterpret_cast<const unsigned char*>(X.text.data());
    const size_t end = X.text.size();
    if (p0 + hs > end) bad("appended offset past the end of the file");
    if (!X.zlib) {
      const uint64_t nbytes = read_uint(base + p0, hs);
      if (p0 + hs + nbytes > end) bad("appended array past the end of the file");
      return std::vector<unsigned char>(base + p0 + hs, base + p0 + hs + nbytes);
    }
    const uint64_t nb = read_uint(base + p0, hs);
    if (p0 + size_t(hs) * (3 + nb) > end) bad("compressed header past the end of the file");
    std::vector<uint64_t> hdr(3 + nb);
    for (size_t k = 0; k < hdr.size(); ++k) hdr[k] = read_uint(base + p0 + k * hs, hs);
    const size_t d0 = p0 + size_t(hs) * (3 + nb);
    return inflate_blocks(hdr, base + d0, end - d0);
  }
  // base64: header and data are encoded as two separate base64 runs
  std::string s;
  size_t pos = 0;
  if (appended) {
    const size_t p0 = X.app_pos + offset;
    size_t e = X.text.find('<', p0);
    if (e == std::string::npos) e = X.text.size();
    s = b64_clean(X.text.data() + p0, e - p0);
  } else {
    s = b64_clean(body.data(), body.size());
  }
  if (!X.zlib) {
    const size_t hl = b64_len(hs);
    if (s.size() >= hl && s[hl - 1] == '=') {  // VTK: the header is its own base64 run
      const auto h = b64_decode(s, pos, hl);
      const uint64_t nbytes = read_uint(h.data(), hs);
      auto d = b64_decode(s, pos + hl, b64_len(nbytes));
      d.resize(nbytes);
      return d;
    }
    // header and data encoded as one run
    const auto h = b64_decode(s, pos, hl);
    const uint64_t nbytes = read_uint(h.data(), hs);
    auto d = b64_decode(s, pos, b64_len(size_t(hs) + nbytes));
    if (d.size() < size_t(hs) + nbytes) bad("truncated base64 data");
    return std::vector<unsigned char>(d.begin() + hs, d.begin() + hs + nbytes);
  }
  const auto h1 = b64_decode(s, pos, b64_len(hs));
  const uint64_t nb = read_uint(h1.data(), hs);
  const size_t hbytes = size_t(hs) * (3 + nb), hl = b64_len(hbytes);
  const auto h = b64_decode(s, pos, hl);
  std::vector<uint64_t> hdr(3 + nb);
  for (size_t k = 0; k < hdr.size(); ++k) hdr[k] = read_uint(h.data() + k * hs, hs);
  uint64_t csum = 0;
  for (uint64_t b = 0; b < nb; ++b) csum += hdr[3 + b];
  const auto d = b64_decode(s, pos + hl, b64_len(csum));
  return inflate_blocks(hdr, d.data(), d.size());
}

std::vector<double> data_array(const XmlFile& X, const std::string& tag, const std::string& body) {
  const std::string fmt = attr(tag, "format"), type = attr(tag, "type");
  std::vector<double> v;
  if (fmt == "ascii") {
    std::istringstream is(body);
    double x;
    while (is >> x) v.push_back(x);
    return v;
  }
  if (fmt != "binary" && fmt != "appended") bad("unsupported DataArray format " + fmt);
  const int ts = type_size(type);
  const bool app = fmt == "appended";
  if (app && X.app_enc.empty()) bad("appended DataArray without AppendedData");
  const size_t off = app ? size_t(std::stoull(attr(tag, "offset"))) : 0;
  const auto bytes = binary_payload(X, app, body, off);
  v.resize(bytes.size() / ts);
  for (size_t k = 0; k < v.size(); ++k) v[k] = as_double(type, bytes.data() + k * ts);
  return v;
}

// The opening tag starting at p (up to '>'), and the element body up to its </DataArray>.
void element(const std::string& t, size_t p, std::string& tag, std::string& body) {
  const size_t e = t.find('>', p);
  if (e == std::string::npos) bad("unterminated tag");
  tag = t.substr(p, e + 1 - p);
  body.clear();
  if (t[e - 1] == '/') return;
  const size_t c = t.find("</DataArray>", e);
  if (c == std::string::npos) bad("DataArray without end tag");
  body = t.substr(e + 1, c - e - 1);
}

void read_vtu(const std::string& path, int nx, double* m, double* time_ps) {
  std::ifstream f(path, std::ios::binary);
  if (!f) bad("file " + path + " not found");
  XmlFile X;
  X.text.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  const std::string& t = X.text;
  // everything before the appended block is XML text
  const size_t ad = t.find("<AppendedData");
  const size_t xml_end = ad == std::string::npos ? t.size() : ad;
  const size_t vf = t.find("<VTKFile");
  if (vf == std::string::npos || vf > xml_end) bad("not a VTK XML file");
  const std::string vtag = t.substr(vf, t.find('>', vf) - vf + 1);
  if (attr(vtag, "type") != "UnstructuredGrid") bad("not an UnstructuredGrid file");
  if (attr(vtag, "byte_order") == "BigEndian") bad("big-endian data is not supported");
  const std::string ht = attr(vtag, "header_type");
  X.hsize = ht == "UInt64" ? 8 : 4;
  const std::string comp = attr(vtag, "compressor");
  if (!comp.empty()) {
    if (comp != "vtkZLibDataCompressor") bad("unsupported compressor " + comp);
    X.zlib = true;
  }
  if (ad != std::string::npos) {
    const std::string atag = t.substr(ad, t.find('>', ad) - ad + 1);
    X.app_enc = attr(atag, "encoding");
    const size_t us = t.find('_', ad + atag.size());
    if (us == std::string::npos) bad("AppendedData without '_' marker");
    X.app_pos = us + 1;
  }
  const size_t piece = t.find("<Piece", vf);
  if (piece == std::string::npos || piece > xml_end) bad("no Piece element");
  const std::string ptag = t.substr(piece, t.find('>', piece) - piece + 1);
  const long long np = std::stoll(attr(ptag, "NumberOfPoints"));
  if (np != nx)
    bad("inconsistent number of points: read " + std::to_string(np) + " but expected " + std::to_string(nx));
  // the time: a field-data array named timeInPs (optional, 0 if absent)
  *time_ps = 0.0;
  const size_t fd = t.find("<FieldData", vf);
  if (fd != std::string::npos && fd < xml_end) {
    const size_t fe = t.find("</FieldData>", fd);
    for (size_t p = t.find("<DataArray", fd); p != std::string::npos && p < fe; p = t.find("<DataArray", p + 1)) {
      std::string tag, body;
      element(t, p, tag, body);
      if (attr(tag, "Name") == "timeInPs") {
        const auto v = data_array(X, tag, body);
        if (!v.empty()) *time_ps = v[0];
      }
    }
  }
  const size_t pd = t.find("<PointData", piece);
  if (pd == std::string::npos || pd > xml_end) bad("no data on the magnetization found in file " + path);
  const size_t pe = t.find("</PointData>", pd);
  for (size_t p = t.find("<DataArray", pd); p != std::string::npos && p < pe; p = t.find("<DataArray", p + 1)) {
    std::string tag, body;
    element(t, p, tag, body);
    if (attr(tag, "Name") != "Magnetization") continue;
    const std::string nc = attr(tag, "NumberOfComponents");
    if (nc != "3") bad("Magnetization must have 3 components");
    const auto v = data_array(X, tag, body);
    if (v.size() != size_t(3) * nx) bad("Magnetization array has the wrong length");
    for (int i = 0; i < nx; ++i)
      for (int d = 0; d < 3; ++d) m[size_t(d) * nx + i] = v[size_t(3) * i + d];
    return;
  }
  bad("no data on the magnetization found in file " + path);
}

// Legacy ASCII .vtk (vtkUnstructuredGridReader's input): POINTS n, then in POINT_DATA either
// "VECTORS Magnetization <type>" or a FIELD array "Magnetization 3 n <type>"; the time from a FIELD
// array "timeInPs 1 1 <type>" anywhere in the file.
void read_vtk_legacy(const std::string& path, int nx, double* m, double* time_ps) {
  std::ifstream f(path);
  if (!f) bad("file " + path + " not found");
  std::string line;
  std::getline(f, line);
  if (line.rfind("# vtk DataFile", 0) != 0) bad("not a legacy VTK file");
  std::getline(f, line);   // title
  std::getline(f, line);
  if (line.find("ASCII") == std::string::npos) bad("only ASCII legacy VTK files are supported");
  *time_ps = 0.0;
  std::string w;
  long long np = -1;
  bool in_point_data = false, found = false;
  auto read_vals = [&](size_t count, std::vector<double>& v) {
    v.resize(count);
    for (size_t k = 0; k < count; ++k)
      if (!(f >> v[k])) bad("truncated data in " + path);
  };
  std::vector<double> vals;
  while (f >> w) {
    if (w == "POINTS") {
      std::string type;
      f >> np >> type;
      if (np != nx)
        bad("inconsistent number of points: read " + std::to_string(np) + " but expected " + std::to_string(nx));
      read_vals(size_t(3) * np, vals);
    } else if (w == "CELLS") {
      long long nc, sz;
      f >> nc >> sz;
      std::getline(f, line);
      std::streampos pos = f.tellg();
      std::getline(f, line);
      if (line.rfind("OFFSETS", 0) == 0) {     // version 5 layout: OFFSETS / CONNECTIVITY blocks
        read_vals(size_t(nc), vals);
        f >> w;
        std::getline(f, line);
        read_vals(size_t(sz), vals);
      } else {                                 // older layout: nc lines "k id_1 .. id_k", sz values in all
        f.seekg(pos);
        read_vals(size_t(sz), vals);
      }
    } else if (w == "CELL_TYPES") {
      long long nc;
      f >> nc;
      read_vals(size_t(nc), vals);
    } else if (w == "POINT_DATA") {
      long long n;
      f >> n;
      in_point_data = true;
    } else if (w == "CELL_DATA") {
      long long n;
      f >> n;
      in_point_data = false;
    } else if (w == "VECTORS" || w == "NORMALS") {
      std::string name, type;
      f >> name >> type;
      read_vals(size_t(3) * (in_point_data ? nx : 0), vals);
      if (in_point_data && name == "Magnetization") {
        for (int i = 0; i < nx; ++i)
          for (int d = 0; d < 3; ++d) m[size_t(d) * nx + i] = vals[size_t(3) * i + d];
        found = true;
      }
    } else if (w == "SCALARS") {
      std::getline(f, line);
      std::istringstream is(line);
      std::string name, type;
      int nc = 1;
      is >> name >> type >> nc;
      f >> w;
      if (w == "LOOKUP_TABLE") f >> w;
      else bad("SCALARS without LOOKUP_TABLE");
      read_vals(size_t(nc) * (in_point_data ? nx : 0), vals);
    } else if (w == "FIELD") {
      std::string name;
      int narr;
      f >> name >> narr;
      for (int a = 0; a < narr; ++a) {
        std::string an, type;
        long long nc, nt;
        f >> an >> nc >> nt >> type;
        read_vals(size_t(nc * nt), vals);
        if (an == "timeInPs" && !vals.empty()) *time_ps = vals[0];
        if (in_point_data && an == "Magnetization" && nc == 3 && nt == nx) {
          for (int i = 0; i < nx; ++i)
            for (int d = 0; d < 3; ++d) m[size_t(d) * nx + i] = vals[size_t(3) * i + d];
          found = true;
        }
      }
    } else if (w == "METADATA") {
      // skip to the blank line that ends the block
      std::getline(f, line);
      while (std::getline(f, line) && !line.empty()) {
      }
    }
  }
  if (np < 0) bad("no POINTS in " + path);
  if (!found) bad("no data on the magnetization found in file " + path);
}

}  // namespace

int read_magnetization(const std::string& path, int nx, double* m, double* time_ps, std::string& err) {
  const size_t dot = path.rfind('.');
  const std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
  try {
    if (ext == "vtu") read_vtu(path, nx, m, time_ps);
    else if (ext == "vtk") read_vtk_legacy(path, nx, m, time_ps);
    else bad("file type " + ext + " not supported");
  } catch (const ReadError& e) {
    err = "read_magnetization: " + e.msg;
    return TMB_ERR_ARG;
  } catch (const std::exception& e) {
    err = std::string("read_magnetization: ") + e.what();
    return TMB_ERR_ARG;
  }
  return TMB_OK;
}

// --------------------------------------------------------------------------------------------
// .log columns
// --------------------------------------------------------------------------------------------
namespace {

// A row vector as Eigen's default formatting prints it with the stream's current flags:
// each coefficient right-aligned to the widest one, one space between them.
void row3(std::ostream& os, const double v[3]) {
  size_t width = 0;
  for (int k = 0; k < 3; ++k) {
    std::ostringstream s;
    s.copyfmt(os);
    s << v[k];
    width = std::max(width, s.str().size());
  }
  for (int k = 0; k < 3; ++k) {
    if (k) os << ' ';
    os << std::setw(int(width)) << v[k];
  }
}

}  // namespace

std::string log_header(const char* start_time, const char* host, const char* user) {
  std::ostringstream o;
  o << "# Log file for simulation started " << (start_time ? start_time : "");
  o << "# on host " << (host ? host : "") << " by user " << (user ? user : "") << "\n";
  o << "# data in the columns is: \n#(1) time in ps, (2) total energy , "
       "(3) demagnetizing energy, (4) exchange energy\n#(5) uniaxial anisotropy energy, "
       "(6) Zeeman energy, (7) cubic anisotropy energy (8) surface anisotropy energy, "
       "\n#(9) bulk DMI energy (10) maximum torque, (11-13) Mx, My, Mz, (14-16) Hx, Hy, Hz. All energies in J/m3, "
       "all fields in T\n";
  return o.str();
}

std::string log_row(double t_ps, const double e[8], double torque, const double mean_m[3], const double mean_h_t[3]) {
  std::ostringstream o;
  o << std::fixed << std::setprecision(4) << t_ps;
  for (int k = 0; k < 8; ++k) o << '\t' << e[k];
  o << '\t' << std::setprecision(3) << std::scientific << torque << '\t' << std::setprecision(10)
    << std::defaultfloat;
  row3(o, mean_m);
  o << '\t' << std::fixed << std::setprecision(6);
  row3(o, mean_h_t);
  o << '\n';
  return o.str();
}

}  // namespace tmb
