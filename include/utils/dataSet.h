// utils/dataSet.h -- C++ drop-in for DynaMap::utils::dataSet (reference
// include/utils/utils_Dataset.h:38-85, utils_Dataset.cpp): the frames of a
// TUM-layout directory (rgb/ and depth/ PNG images named by time stamp, an
// optional association file, an optional groundtruth.txt) in time order,
// as the session's inputs -- raw uint16 depth and RGB bytes.  Header-only;
// link with -lz.
//
// Differences from the reference, each a fix: depth is read as 16 bits (the
// reference reads it with cv::IMREAD_COLOR, utils_Dataset.cpp:233-235, which
// drops it to 8 bits); RGB comes in RGB order; association.txt is used when
// present (the reference never sets assciateFileExist, :16-52) and read by
// its paths, so either column order works (the reference takes word 0 as
// depth and word 2 as RGB, :174-175); a frame's ground truth is the line
// nearest in time (within 0.02 s) rather than line curID +
// offsetLineGroundTruth, an offset the reference leaves unset (:210-221);
// getCurrentPose() without ground truth is the identity rather than an
// uninitialised matrix (:69-88).  OpenCV is absent, so the
// PNG reader below decodes what TUM recordings use: non-interlaced 8-bit
// grey / RGB / RGBA and 16-bit grey, every filter type (zlib inflates).
#pragma once

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../dynamap/pose_io.h"
#include "../dynamap/types.h"

namespace DynaMap {
namespace utils {

namespace png {

struct Image {
  int rows = 0, cols = 0, channels = 0, bits = 0;  // channels 1, 3 or 4; bits 8 or 16
  std::vector<uint8_t> data;                        // unfiltered rows, PNG byte order
};

inline uint32_t be32(const uint8_t* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

// PNG (ISO/IEC 15948) reader for the formats above.
inline Image read(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<uint8_t> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (b.size() < 8 || !std::equal(sig, sig + 8, b.begin()))
    throw std::runtime_error(path + ": not a PNG file");
  Image im;
  int color = -1, interlace = 0;
  std::vector<uint8_t> z;
  size_t pos = 8;
  while (pos + 12 <= b.size()) {
    const uint32_t len = be32(&b[pos]);
    const std::string type(b.begin() + pos + 4, b.begin() + pos + 8);
    if (pos + 12 + (size_t)len > b.size()) throw std::runtime_error(path + ": truncated");
    const uint8_t* d = &b[pos + 8];
    if (type == "IHDR") {
      im.cols = (int)be32(d);
      im.rows = (int)be32(d + 4);
      im.bits = d[8];
      color = d[9];
      interlace = d[12];
    } else if (type == "IDAT") {
      z.insert(z.end(), d, d + len);
    } else if (type == "IEND") {
      break;
    }
    pos += 12 + (size_t)len;
  }
  im.channels = color == 0 ? 1 : color == 2 ? 3 : color == 6 ? 4 : 0;
  if (im.channels == 0 || interlace != 0 || (im.bits != 8 && im.bits != 16) ||
      (im.bits == 16 && im.channels != 1) || im.rows <= 0 || im.cols <= 0)
    throw std::runtime_error(path + ": unsupported PNG format");
  const size_t bpp = (size_t)im.channels * (im.bits / 8);
  const size_t stride = bpp * (size_t)im.cols;
  std::vector<uint8_t> raw((stride + 1) * (size_t)im.rows);
  uLongf raw_len = (uLongf)raw.size();
  if (uncompress(raw.data(), &raw_len, z.data(), (uLong)z.size()) != Z_OK ||
      raw_len != raw.size())
    throw std::runtime_error(path + ": bad image data");
  im.data.assign(stride * (size_t)im.rows, 0);
  for (int r = 0; r < im.rows; ++r) {
    const uint8_t ft = raw[(stride + 1) * (size_t)r];
    const uint8_t* s = &raw[(stride + 1) * (size_t)r + 1];
    uint8_t* o = &im.data[stride * (size_t)r];
    const uint8_t* up = r ? &im.data[stride * (size_t)(r - 1)] : nullptr;
    for (size_t i = 0; i < stride; ++i) {
      const int a = i >= bpp ? o[i - bpp] : 0;
      const int u = up ? up[i] : 0;
      const int c = (up && i >= bpp) ? up[i - bpp] : 0;
      int pred = 0;
      switch (ft) {
        case 0: pred = 0; break;
        case 1: pred = a; break;
        case 2: pred = u; break;
        case 3: pred = (a + u) / 2; break;
        case 4: {  // Paeth predictor
          const int p = a + u - c, pa = std::abs(p - a), pb = std::abs(p - u),
                    pc = std::abs(p - c);
          pred = (pa <= pb && pa <= pc) ? a : (pb <= pc ? u : c);
          break;
        }
        default: throw std::runtime_error(path + ": bad filter type");
      }
      o[i] = (uint8_t)(s[i] + pred);
    }
  }
  return im;
}

}  // namespace png

// The reference's frame holds cv::Mat depth and rgb; here the session's
// inputs.
struct frame {
  int rows = 0, cols = 0;
  std::vector<uint16_t> depth;  // rows * cols, sensor units (TUM: 5000 per metre)
  std::vector<uint8_t> rgb;     // rows * cols * 3, RGB; empty without an RGB image
  // depth in metres, as the reference's frame holds it (:236)
  std::vector<float> depthMetres(float depthScaler) const {
    std::vector<float> m(depth.size());
    for (size_t i = 0; i < depth.size(); ++i) m[i] = (float)depth[i] * (1.0f / depthScaler);
    return m;
  }
};

class dataSet {
 public:
  std::string rgbFolderAddress;
  std::string depthFolderAddress;
  std::string groundTruthFileAddress;
  std::string associationFileAddress;
  std::vector<std::string> depthFileNames;  // paths, in time order
  std::vector<std::string> rgbFileNames;    // paired with depthFileNames ("" if none)
  // file names are prefix + time stamp (or frame number) + suffix
  // (utils_Dataset.cpp:40-48: TUM "" / ".png"; other layouts "depth_",
  // "color_"); set them and call loadData() again to re-list
  std::string depthPrefix;
  std::string rgbPrefix;
  std::string depthSuffix = ".png";
  std::string rgbSuffix = ".png";
  std::size_t firstFrameID = 0;  // kept for the reference's callers; unused there too
  std::size_t lastFrameID = 0;
  std::size_t skipFrameNum = 0;
  std::size_t curID = 0;
  rgbdSensor sensor;             // depthScaler for depthMetres()
  bool groundTruthExist = false;
  bool assciateFileExist = false;
  std::vector<std::string> refLines;       // ground-truth lines (no comments)
  std::vector<double> groundTruthLine;     // of the frame last read (8 values) or empty
  double stamp = 0.0;                      // depth time stamp of the frame last read
  frame image;

  // utils_Dataset.cpp:13-54
  explicit dataSet(std::string mainDir) : mainDir_(std::move(mainDir)) {
    rgbFolderAddress = mainDir_ + "/rgb/";
    depthFolderAddress = mainDir_ + "/depth/";
    groundTruthFileAddress = mainDir_ + "/groundtruth.txt";
    associationFileAddress = mainDir_ + "/association.txt";
    loadData();
  }
  virtual ~dataSet() = default;

  // utils_Dataset.cpp:58-68: the frame list and the ground-truth lines
  bool loadData() {
    namespace fs = std::filesystem;
    const std::string& mainDir = mainDir_;
    depthFileNames.clear();
    rgbFileNames.clear();
    assciateFileExist = fs::exists(associationFileAddress);
    if (assciateFileExist) {
      std::ifstream in(associationFileAddress);
      std::string ln;
      std::vector<std::pair<std::string, std::string>> pairs;
      while (std::getline(in, ln)) {
        if (ln.empty() || ln[0] == '#') continue;
        std::istringstream ss(ln);
        std::string t0, p0, t1, p1;
        if (!(ss >> t0 >> p0 >> t1 >> p1)) continue;
        if (p0.rfind("depth", 0) == 0) pairs.push_back({mainDir + "/" + p0, mainDir + "/" + p1});
        else pairs.push_back({mainDir + "/" + p1, mainDir + "/" + p0});
      }
      std::stable_sort(pairs.begin(), pairs.end(), [&](const auto& x, const auto& y) {
        return file_stamp(x.first, depthPrefix, depthSuffix) <
               file_stamp(y.first, depthPrefix, depthSuffix);
      });
      for (auto& p : pairs) {
        depthFileNames.push_back(p.first);
        rgbFileNames.push_back(p.second);
      }
    } else {
      depthFileNames = invokeFileNames(depthFolderAddress, depthSuffix, depthPrefix);
      std::vector<std::string> rgb = fs::is_directory(rgbFolderAddress)
                                         ? invokeFileNames(rgbFolderAddress, rgbSuffix, rgbPrefix)
                                         : std::vector<std::string>();
      rgb.resize(depthFileNames.size());  // paired by index, as the reference
      rgbFileNames = rgb;
    }
    refLines = getFileContent(groundTruthFileAddress);
    return true;
  }

  // utils_Dataset.cpp:111-148: the files prefix*suffix of a folder, ordered
  // by the number between prefix and suffix (paths)
  static std::vector<std::string> invokeFileNames(const std::string& folder,
                                                  const std::string& suffix = ".png",
                                                  const std::string& prefix = "") {
    std::vector<std::string> names;
    for (const auto& e : std::filesystem::directory_iterator(folder)) {
      const std::string f = e.path().filename().string();
      if (f.size() > prefix.size() + suffix.size() && f.compare(0, prefix.size(), prefix) == 0 &&
          f.compare(f.size() - suffix.size(), suffix.size(), suffix) == 0)
        names.push_back(e.path().string());
    }
    std::stable_sort(names.begin(), names.end(), [&](const std::string& a, const std::string& b) {
      return file_stamp(a, prefix, suffix) < file_stamp(b, prefix, suffix);
    });
    return names;
  }

  // utils_Dataset.cpp:182-209: the non-comment lines of a file
  std::vector<std::string> getFileContent(const std::string& fileName) {
    std::vector<std::string> out;
    std::ifstream in(fileName);
    groundTruthExist = (bool)in;
    std::string ln;
    while (in && std::getline(in, ln))
      if (!ln.empty() && ln[0] != '#') out.push_back(ln);
    return out;
  }

  std::size_t size() const { return depthFileNames.size(); }

  // utils_Dataset.cpp:223-242: read frame curID and its ground truth, then
  // advance
  void invokeNextFrame() {
    if (curID >= depthFileNames.size()) throw std::out_of_range("dataSet: no more frames");
    invokeNextImage();
    invokeNextGroundTruthLine();
    ++curID;
  }
  void invokeNextImage() {
    const png::Image d = png::read(depthFileNames[curID]);
    if (d.channels != 1 || d.bits != 16)
      throw std::runtime_error(depthFileNames[curID] + ": depth must be 16-bit grey");
    image.rows = d.rows;
    image.cols = d.cols;
    image.depth.resize((size_t)d.rows * d.cols);
    for (size_t i = 0; i < image.depth.size(); ++i)
      image.depth[i] = (uint16_t)((d.data[2 * i] << 8) | d.data[2 * i + 1]);  // big endian
    stamp = file_stamp(depthFileNames[curID], depthPrefix, depthSuffix);
    image.rgb.clear();
    if (!rgbFileNames[curID].empty()) {
      const png::Image c = png::read(rgbFileNames[curID]);
      if (c.bits != 8 || c.rows != d.rows || c.cols != d.cols)
        throw std::runtime_error(rgbFileNames[curID] + ": RGB must be 8-bit, depth-sized");
      image.rgb.resize((size_t)c.rows * c.cols * 3);
      for (size_t i = 0; i < (size_t)c.rows * c.cols; ++i)
        for (int k = 0; k < 3; ++k)
          image.rgb[3 * i + k] = c.data[i * c.channels + (c.channels == 1 ? 0 : k)];
    }
  }
  // the ground-truth line nearest in time to the frame (within 0.02 s; the
  // earlier line on a tie)
  void invokeNextGroundTruthLine() {
    groundTruthLine.clear();
    if (gt_.size() != refLines.size()) parse_ground_truth();
    auto it = std::lower_bound(gt_order_.begin(), gt_order_.end(), stamp,
                               [&](size_t i, double t) { return gt_[i][0] < t; });
    double best = 0.02;
    for (auto c : {it - (it != gt_order_.begin() ? 1 : 0), it}) {
      if (c == gt_order_.end()) continue;
      const std::vector<double>& v = gt_[*c];
      const double dt = std::fabs(v[0] - stamp);
      if (dt < best || (dt == best && !groundTruthLine.empty() && v[0] < groundTruthLine[0])) {
        best = dt;
        groundTruthLine = v;
      }
    }
  }
  // utils_Dataset.cpp:69-88 (as builder::v2tRef): identity without ground truth
  Matrix4f getCurrentPose() const {
    if (groundTruthLine.size() < 8) return Matrix4f::Identity();
    float p[16];
    pose_io::pose_from_tum(groundTruthLine.data(), p);
    return Matrix4f::from_row_major(p);
  }
  // utils_Dataset.cpp:89-110: overwrite the ground-truth translation
  void setCurrentPose(const Matrix4f& pose) {
    if (groundTruthLine.size() < 8) return;
    groundTruthLine[1] = pose(0, 3);
    groundTruthLine[2] = pose(1, 3);
    groundTruthLine[3] = pose(2, 3);
  }

 private:
  // refLines parsed once: the lines with 8 values, ordered by time stamp
  void parse_ground_truth() {
    gt_.assign(refLines.size(), std::vector<double>());
    gt_order_.clear();
    for (size_t i = 0; i < refLines.size(); ++i) {
      std::istringstream ss(refLines[i]);
      double x;
      while (ss >> x) gt_[i].push_back(x);
      if (gt_[i].size() >= 8) gt_order_.push_back(i);
    }
    std::stable_sort(gt_order_.begin(), gt_order_.end(),
                     [&](size_t a, size_t b) { return gt_[a][0] < gt_[b][0]; });
  }

  std::vector<std::vector<double>> gt_;
  std::vector<size_t> gt_order_;
  std::string mainDir_;
  // the number in a file name between prefix and suffix
  static double file_stamp(const std::string& path, const std::string& prefix,
                           const std::string& suffix) {
    std::string f = std::filesystem::path(path).filename().string();
    if (f.compare(0, prefix.size(), prefix) == 0) f.erase(0, prefix.size());
    if (f.size() >= suffix.size() && f.compare(f.size() - suffix.size(), suffix.size(), suffix) == 0)
      f.erase(f.size() - suffix.size());
    return std::strtod(f.c_str(), nullptr);
  }
};

}  // namespace utils
}  // namespace DynaMap
