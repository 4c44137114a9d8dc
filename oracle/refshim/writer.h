// writer.h stand-in (TEST INFRASTRUCTURE, see qshim.h): no output files.
#pragma once
#include "qshim.h"
namespace LangmuirCore {
class World;
class ChargeAgent;
class Logger : public QObject {
public:
    Logger(World&, QObject* parent = 0) : QObject(parent) {}
    void reportCarrier(ChargeAgent&) {}
    void reportFluxStream() {}
    void saveCoulombEnergy() {}
    void reportXYZStream() {}
};
}  // namespace LangmuirCore
