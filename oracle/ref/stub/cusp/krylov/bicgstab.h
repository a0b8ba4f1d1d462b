#pragma once
#include "../stub.h"
