#pragma once
namespace medyan { struct Filament {}; }
