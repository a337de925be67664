// EDXUtil/Core/Assertion.h includes <Assert.h> (a case-insensitive file system)
#pragma once
#include <assert.h>
