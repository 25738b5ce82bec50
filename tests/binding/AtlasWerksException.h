// stand-in: AtlasWerksException (Base/AtlasWerksException.h)
#pragma once
#include <stdexcept>
#include <string>
class AtlasWerksException : public std::runtime_error {
 public:
  AtlasWerksException(const char *file, int line, const std::string &msg)
      : std::runtime_error(std::string(file) + ":" + std::to_string(line) + ": " + msg) {}
};
