// Stands in for EDXUtil/Windows/Debug.h, whose explicit specialisations in
// class scope g++ rejects. It keeps that header's includes; a release build
// (no _DEBUG) never calls the debugging helpers it declares
// (EDXUtil/Core/Assertion.h:38-42).
#pragma once
#include "Base.h"
#include "../Core/Types.h"
namespace EDX {
class Debug {};
}
