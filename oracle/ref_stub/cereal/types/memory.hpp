// cereal stub: see archives/binary.hpp
#pragma once
#include <memory>
