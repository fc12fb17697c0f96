// image/sensor/rgbdImage.h -- the frame handed to the C++ drop-in classes,
// standing in for DynaMap::rgbdImage (reference
// include/image/sensor/rgbdImage.h:37-66).  The reference's image holds
// managed float depth; here it points at the sensor's host frame: uint16
// depth in sensor units (metres * depthScaler) and optional uint8 RGB.
#pragma once

#include <cstdint>

#include "../../dynamap/types.h"

namespace DynaMap {

struct rgbdImage {
  rgbdSensor sensor;
  const uint16_t* depth = nullptr;  // rows*cols, row-major, 0 = invalid
  const uint8_t* rgb = nullptr;     // rows*cols*3 R,G,B or null

  void init(const rgbdSensor& s) { sensor = s; }
};

}  // namespace DynaMap
