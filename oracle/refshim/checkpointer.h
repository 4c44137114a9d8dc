// checkpointer.h stand-in (TEST INFRASTRUCTURE, see qshim.h): the harness
// builds worlds from parameters, never from a file.
#pragma once
#include "qshim.h"
#include "parameters.h"
namespace LangmuirCore {
class World;
class CheckPointer : public QObject {
public:
    explicit CheckPointer(World&, QObject* parent = 0) : QObject(parent) {}
    void load(const QString&, ConfigurationInfo&) {
        qFatal("refshim: checkpoint files are not read by the harness");
    }
    void save(const QString& = "") {}
};
}  // namespace LangmuirCore
