// Drop-in for the reference's image.h (image.h:10-91): float RGB image,
// row-major (index 3j + 3*width*i), PPM (P3) output.
#ifndef PM_DROPIN_IMAGE_H
#define PM_DROPIN_IMAGE_H
#include <algorithm>
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "core.h"

class Image {
  unsigned int width, height;
  std::vector<float> pixels;
  unsigned int index(unsigned int i, unsigned int j) const { return 3 * j + 3 * width * i; }

 public:
  Image(unsigned int width, unsigned int height) : width(width), height(height) {
    pixels.resize(3 * width * height);
  }
  unsigned int getWidth() const { return width; }
  unsigned int getHeight() const { return height; }
  float* data() { return pixels.data(); }

  Vec3f getPixel(unsigned int i, unsigned int j) const {
    const unsigned int k = index(i, j);
    return Vec3f(pixels[k], pixels[k + 1], pixels[k + 2]);
  }
  void addPixel(unsigned int i, unsigned int j, const Vec3f& rgb) {
    const unsigned int k = index(i, j);
    for (int c = 0; c < 3; ++c) pixels[k + c] += rgb[c];
  }
  void setPixel(unsigned int i, unsigned int j, const Vec3f& rgb) {
    const unsigned int k = index(i, j);
    for (int c = 0; c < 3; ++c) pixels[k + c] = rgb[c];
  }
  void divide(const float k) {
    for (unsigned int i = 0; i < height; ++i)
      for (unsigned int j = 0; j < width; ++j) setPixel(i, j, getPixel(i, j) / k);
  }
  void gammaCorrection(const float gamma) {
    for (float& p : pixels) p = std::pow(p, 1.0f / gamma);
  }
  void writePPM(const std::string& filename) {
    std::ofstream f(filename);
    f << "P3\n" << width << " " << height << "\n255\n";
    for (unsigned int i = 0; i < height; ++i)
      for (unsigned int j = 0; j < width; ++j) {
        const Vec3f c = getPixel(i, j);
        for (int k = 0; k < 3; ++k) {
          const unsigned int q = std::clamp(static_cast<unsigned int>(255.0f * c[k]), 0u, 255u);
          f << q << (k < 2 ? " " : "\n");
        }
      }
  }
};

#endif
